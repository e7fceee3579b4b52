// Drop-in for the reference's stability Worker (src/stabworker.js): the same message
// protocol -- request {key, points: [{S, modal}], tool, mat, arc, fz, nonlinear}, replies
// {key, S, alim, open} per point then {key, done: true}; a newer request replaces an older
// one.  The whole sweep is one GPU job; a newer request cancels the older job on the
// device at its next trial boundary.  Runs as a Node worker_threads worker or, in an
// Electron renderer's Worker, with the Web Worker `self` interface.
import { timeDomainLimits, cancelSweeps } from './stabtd.js';

let parentPort = null;
try {
  ({ parentPort } = await import('node:worker_threads'));
} catch {
  parentPort = null;
}
const post = (m) => (parentPort ? parentPort.postMessage(m) : self.postMessage(m));

let job = 0;
async function onRequest(m) {
  const id = ++job;
  cancelSweeps(); // the older request's job stops at its next trial boundary
  let res;
  try {
    res = await timeDomainLimits(m.tool, m.mat, m.arc, m.fz, m.points, { nonlinear: m.nonlinear });
  } catch (e) {
    if (id !== job || e.code === 'MCS_ERR_CANCELLED') return; // replaced by a newer request
    throw e;
  }
  for (const r of res) {
    if (id !== job) return;
    post({ key: m.key, S: r.S, alim: r.alim, open: r.open });
  }
  if (id === job) post({ key: m.key, done: true });
}

if (parentPort) parentPort.on('message', onRequest);
else self.onmessage = ({ data }) => onRequest(data);
