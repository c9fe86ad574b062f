"""Build libchaoslab_b200.so in-tree for sm_100a (and nothing else).

Every translation unit is compiled by nvcc with `-gencode arch=compute_100a,code=sm_100a -fmad=false`: the orbit
kernels reproduce the reference's Float64 rounding operation for operation, so nothing may be contracted into an fma
behind the source's back (the kernels write their fmas explicitly). Objects go to chaos_b200/_build/ and are
rebuilt only when a source or header is newer; the library lands next to this file.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchaoslab_b200.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(path: str, seen: set | None = None) -> set:
    """The project headers `path` includes, transitively (quoted includes resolved beside the file, in csrc/ and in
    include/)."""
    seen = set() if seen is None else seen
    try:
        text = open(path).read()
    except OSError:
        return seen
    for name in _INCLUDE.findall(text):
        for base in (os.path.dirname(path), CSRC, os.path.join(ROOT, "include")):
            cand = os.path.normpath(os.path.join(base, name))
            if os.path.exists(cand):
                if cand not in seen:
                    seen.add(cand)
                    _deps(cand, seen)
                break
    return seen


def _compile(src: str, verbose_ptxas: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _deps(src)])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest and not verbose_ptxas:
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(jobs: int | None = None, verbose_ptxas: bool = False) -> str:
    sys.path.insert(0, CSRC)
    try:
        import gen_menu  # noqa: WPS433
        gen_menu.main()
    finally:
        sys.path.pop(0)
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    # the biggest units first, so the parallel build ends together
    srcs.sort(key=lambda p: -os.path.getsize(p))
    jobs = jobs or max(1, os.cpu_count() or 1)
    logs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = [f.result() for f in [ex.submit(_compile, s, verbose_ptxas) for s in srcs]]
    objs, logs = [o for o, _ in objs], [l for _, l in objs if l]
    newest = max(os.path.getmtime(o) for o in objs)
    stale = {os.path.join(BUILD, fn) for fn in os.listdir(BUILD)} - set(objs)
    for s in stale:
        if s.endswith(".o"):
            os.remove(s)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
