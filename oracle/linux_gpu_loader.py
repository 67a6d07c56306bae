"""Writes a copy of the reference's src/integrators/gpu_path.cpp whose module loader has a Linux
branch: where the reference reports "GPU rendering is only available on Windows builds", the copy
dlopen()s libprender_gpu.so (beside the executable, else on the loader's search path) and
resolves the same three entry points with the same version check as the Windows branch
(gpu_path.cpp:45-74). This is the binding INTEGRATION.md describes; nothing else in the file
changes. TEST INFRASTRUCTURE (oracle/Makefile's `prender` target): the reference file is read
where it lies and the copy is written under oracle/_ref/.

    python3 linux_gpu_loader.py <reference gpu_path.cpp> <output gpu_path.cpp>
"""

import sys

LINUX_BRANCH = """#else
        std::string dir = std::filesystem::canonical("/proc/self/exe").parent_path().string();
        void *h = dlopen((dir + "/libprender_gpu.so").c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!h) h = dlopen("libprender_gpu.so", RTLD_NOW | RTLD_LOCAL);
        if (!h) {
            const char *why = dlerror();
            g.status = std::string("libprender_gpu.so not found: ") + (why ? why : "");
            return g;
        }
        auto version = reinterpret_cast<int (*)()>(dlsym(h, "prgpu_api_version"));
        g.listDevices = reinterpret_cast<decltype(g.listDevices)>(dlsym(h, "prgpu_list_devices"));
        g.render = reinterpret_cast<decltype(g.render)>(dlsym(h, "prgpu_render"));
        if (!version || !g.listDevices || !g.render || version() != prgpu::kApiVersion) {
            g.status = "libprender_gpu.so has an incompatible interface";
            return g;
        }
        g.loaded = true;
        g.status = "ok";
#endif"""

WINDOWS_ONLY = '        g.status = "GPU rendering is only available on Windows builds";\n#endif'


def main():
    src_path, out_path = sys.argv[1], sys.argv[2]
    with open(src_path) as f:
        src = f.read()
    i = src.find(WINDOWS_ONLY)
    if i < 0 or src.find(WINDOWS_ONLY, i + 1) >= 0:
        raise SystemExit("gpu_path.cpp: the loader's non-Windows branch was not found exactly once")
    j = src.rfind("#else", 0, i)
    if j < 0 or src[j:i].strip() != "#else":
        raise SystemExit("gpu_path.cpp: unexpected text before the non-Windows branch")
    out = "#ifndef _WIN32\n#include <dlfcn.h>\n#endif\n" + src[:j] + LINUX_BRANCH + src[i + len(WINDOWS_ONLY):]
    with open(out_path, "w") as f:
        f.write(out)


if __name__ == "__main__":
    main()
