# node-gyp build of the addon: `node-gyp rebuild` in this directory, after libwt.so is built
# (python -m windtunnel_vis_b200.build). The addon finds libwt.so through its rpath.
{
  "targets": [
    {
      "target_name": "wt_napi",
      "sources": ["wt_napi.c", "wt_addon.c"],
      "include_dirs": ["../include", "."],
      "libraries": ["-L<(module_root_dir)/../windtunnel_vis_b200", "-lwt", "-lm",
                    "-Wl,-rpath,<(module_root_dir)/../windtunnel_vis_b200"],
      "cflags": ["-std=c99", "-O2", "-Wall"]
    }
  ]
}
