{
  "targets": [
    {
      "target_name": "gsb200",
      "sources": ["gsb200_addon.cc"],
      "include_dirs": ["../../include"],
      "cflags_cc": ["-std=c++17", "-O2"],
      "libraries": ["-L<(module_root_dir)/..", "-lgsb200", "-Wl,-rpath,<(module_root_dir)/.."],
      "defines": ["NAPI_VERSION=8"]
    }
  ]
}
