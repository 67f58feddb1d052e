"""Build recipe for the in-tree CUDA library ``seqtree_b200/libseqtree_b200.so``.

Every ``csrc/*.cu`` and ``csrc/*.cpp`` file is compiled for sm_100a only and linked into one
shared library with the CUDA runtime linked statically, so the ``.so`` travels with the source
tree and needs nothing from a JIT cache.  Objects go to ``seqtree_b200/_build/``; a file is
recompiled only when it or a header is newer than its object.

    python -m seqtree_b200.build            # build (incremental)
    python -m seqtree_b200.build --force    # rebuild everything
    python -m seqtree_b200.build --verbose  # also print ptxas register/spill reports
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libseqtree_b200.so"
INCLUDE = HERE.parent / "include"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
           f"-I{INCLUDE}"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", f"-I{INCLUDE}", "-I/usr/local/cuda/include"]


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc")) + \
        list(INCLUDE.rglob("*.h")) + list(INCLUDE.rglob("*.hpp"))


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def build_pack(force: bool = False) -> Path:
    """The CPython extension ``seqtree_b200._pack`` (``csrc/pack_py.c``), which packs the Python
    mirror's string lists; built with the running interpreter's headers."""
    import sysconfig
    src = CSRC / "pack_py.c"
    out = HERE / ("_pack" + sysconfig.get_config_var("EXT_SUFFIX"))
    if force or not out.exists() or src.stat().st_mtime > out.stat().st_mtime:
        cmd = ["gcc", "-O2", "-shared", "-fPIC", f"-I{sysconfig.get_paths()['include']}",
               str(src), "-o", str(out)]
        print("[seqtree_b200]", "gcc", src.name, flush=True)
        subprocess.run(cmd, check=True)
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    build_pack(force)
    BUILD.mkdir(exist_ok=True)
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objs = []
    for src in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and not _stale(obj, src, newest):
            continue
        if src.suffix == ".cu":
            cmd = [NVCC, *ARCH, *CUFLAGS, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        else:
            cmd = ["g++", *CXXFLAGS, "-c", str(src), "-o", str(obj)]
        print("[seqtree_b200]", " ".join(cmd[:1] + [src.name]), flush=True)
        subprocess.run(cmd, check=True)
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
               "-lpthread"]
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(args.force, args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
