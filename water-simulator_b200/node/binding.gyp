{
  "targets": [
    {
      "target_name": "swe_napi",
      "sources": ["swe_napi.cc"],
      "include_dirs": ["../../include"],
      "cflags_cc": ["-std=c++17", "-O2"],
      "cflags_cc!": ["-fno-exceptions"],
      "libraries": ["-L<(module_root_dir)/..", "-lswe_b200", "-Wl,-rpath,<(module_root_dir)/.."]
    }
  ]
}
