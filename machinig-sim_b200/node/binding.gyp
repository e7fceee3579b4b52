{
  "targets": [
    {
      "target_name": "mcs",
      "sources": ["mcs_napi.c"],
      "include_dirs": ["../../include"],
      "defines": ["MCS_HAVE_NODE_API_H", "NAPI_VERSION=8"],
      "libraries": ["-L<(module_root_dir)/..", "-lmcs", "-Wl,-rpath,<(module_root_dir)/.."]
    }
  ]
}
