// Drop-in for the reference's src/stabtd.js (and the lobe read-out of src/sld.js) on
// Node/Electron hosts: the same exported names, arguments and return shapes, computed by
// libmcs.so on the GPU through the mcs.node addon.
//   import { timeDomainLimit, chatterAt } from './stabtd.js';
import { createRequire } from 'node:module';

const require = createRequire(import.meta.url);
const addon = require('./build/Release/mcs.node');

// stabtd.js:14 -- one trial: true when the chatter index exceeds 0.45
export function chatterAt(tool, modal, mat, S, arc, fz, ap, opts = {}) {
  return addon.chatterAt(tool, modal, mat, S, arc, fz, ap, opts);
}

// stabtd.js:24 -- { alim, bracket: [stable, chatter] }, bracket[1] === Infinity when open
export function timeDomainLimit(tool, modal, mat, S, arc, fz, opts = {}) {
  return addon.timeDomainLimit(tool, modal, mat, S, arc, fz, opts);
}

// the Worker's sweep (stabworker.js:8-13) as one GPU job: [{ S, alim, open }]
export function timeDomainLimits(tool, mat, arc, fz, points, opts = {}) {
  return addon.timeDomainLimits(tool, mat, arc, fz, points, opts);
}

export function cancelSweeps() {
  return addon.cancelSweeps();
}

// alimAt(stabilityLobes(params), rpm) for every rpm (sld.js:23,64)
export function lobeLimit(params, rpms) {
  return addon.lobeLimit(params, Array.from(rpms));
}

export const chatterIndex = (...a) => addon.chatterIndex(...a);
