"""Build recipe for libcastro_b200.so (sm_100a) and its exact-arithmetic twin.

``python build.py`` compiles every CUDA translation unit of ``csrc/`` with nvcc
for sm_100a and links two shared libraries into ``lib/``:

* ``libcastro_b200.so``       -- the production build (FMA contraction on,
                                 factored table interpolation);
* ``libcastro_b200_exact.so`` -- ``-DCASTRO_EXACT --fmad=false``: the
                                 reference's operation order everywhere, used
                                 to show bit-for-bit agreement with a
                                 non-contracting CPU build.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["castro_host.cu", "castro_abi.cu", "castro_sim.cu", "castro_adjoint.cu", "castro_main.cu", "castro_peak.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-Wno-subobject-linkage"]
VARIANTS = {
    "libcastro_b200.so": [],
    "libcastro_b200_exact.so": ["-DCASTRO_EXACT", "--fmad=false"],
}


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "castro_b200.h")]


def _stale(out: str) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in _deps())


def _compile(src: str, obj: str, extra: list[str], verbose: bool) -> None:
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False, variants=None) -> list[str]:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    outs = []
    jobs = []
    names = list(VARIANTS) if variants is None else variants
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for name in names:
            out = os.path.join(LIBDIR, name)
            outs.append(out)
            if not force and not _stale(out):
                continue
            tag = name.replace(".so", "")
            objs = [os.path.join(OBJDIR, f"{tag}_{s.replace('.cu', '.o')}") for s in SOURCES]
            futs = [ex.submit(_compile, s, o, VARIANTS[name], verbose) for s, o in zip(SOURCES, objs)]
            jobs.append((out, objs, futs))
        for out, objs, futs in jobs:
            for f in futs:
                f.result()
            cmd = [NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed for {out}:\n{r.stdout}\n{r.stderr}")
    exe = os.path.join(LIBDIR, "castro_b200.ex")
    if "libcastro_b200.so" in names and (force or _stale(exe)):
        main = os.path.join(OBJDIR, "exe_main.cu")
        with open(main, "w") as fp:
            fp.write('extern "C" int castro_main(int, char**);\nint main(int c, char** v) { return castro_main(c, v); }\n')
        cmd = [NVCC, *ARCH, "-o", exe, main, "-L" + LIBDIR, "-lcastro_b200", "-Xlinker", "-rpath=$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed for {exe}:\n{r.stdout}\n{r.stderr}")
        outs.append(exe)
    # host-only check of the reverse-mode stages against finite differences
    st = os.path.join(LIBDIR, "castro_adjoint_selftest")
    if "libcastro_b200.so" in names and (force or _stale(st)):
        cmd = [NVCC, *ARCH, "-O2", "-std=c++17", "-Xcompiler", "-Wno-subobject-linkage", "-o", st,
               os.path.join(CSRC, "adjoint_selftest.cu")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"build failed for {st}:\n{r.stdout}\n{r.stderr}")
        outs.append(st)
    return outs


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
