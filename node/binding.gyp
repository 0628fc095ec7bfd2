{
  "targets": [
    {
      "target_name": "wsort",
      "sources": ["wsort_node.cc"],
      "include_dirs": ["../include"],
      "libraries": ["-L<(module_root_dir)/../winding_b200", "-lwsort", "-Wl,-rpath,<(module_root_dir)/../winding_b200"],
      "cflags_cc": ["-std=c++17", "-O2"]
    }
  ]
}
