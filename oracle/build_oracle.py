"""Build recipe for the oracle libraries.

Two things are built here, both test infrastructure only:

1. ``oracle/liboracle.so`` from ``oracle/highreg_oracle.c``: the plain-C
   restatement of the reference's hot-path algorithm (the oracle that the GPU
   parity tests compare against). Built with ``gcc -O2`` and no ``-march`` so
   that, like the reference built the same way, no fused multiply-adds are
   emitted and the scalar arithmetic follows the reference's operation order.

2. ``oracle/_ref/*.so``: the UNMODIFIED reference sources compiled where they
   lie (highreg_stokes_2surf/*.cpp and highreg_stokes_extend_to_grid/*.cpp),
   each with a small extern "C" wrapper (``ref_wrap_2s.cpp``,
   ``ref_wrap_e2g.cpp``). The reference sets its treecode parameters P and N0
   as compile-time constants in KITC.h (its README tells users to edit them), so
   each (P, N0) variant is compiled from a scratch copy under /tmp with those two
   constants changed; nothing is copied into this repository. FFTW (absent
   here) is replaced by the test-only header ``fftw_standin/fftw3.h``.

``oracle/_ref`` is git-ignored but travels with the working tree, so the
oracle can use it wherever it was built; the reference tree itself is only
read at build time.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")


def reference_root(path: str | None = None) -> str | None:
    """The reference source tree: ``path`` if given, else $HR_REFERENCE_ROOT,
    else a directory named ``reference`` beside this repository's root. An
    explicitly named tree that does not exist is an error; the default one may
    be absent (machines that only run the prebuilt files), and then None."""
    explicit = path or os.environ.get("HR_REFERENCE_ROOT")
    if explicit:
        if not os.path.isdir(os.path.join(explicit, "highreg_stokes_2surf")):
            raise FileNotFoundError("reference tree not found at %s (HR_REFERENCE_ROOT / argument)" % explicit)
        return explicit
    default = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
    return default if os.path.isdir(os.path.join(default, "highreg_stokes_2surf")) else None


# (P, N0) treecode variants of the reference two-surface program.
KITC_VARIANTS = [(6, 1000), (6, 2000), (4, 300), (10, 8000), (8, 4000)]

CXXFLAGS = ["-std=c++14", "-O2", "-fopenmp", "-fPIC", "-shared", "-w", "-Wl,-Bsymbolic"]


def _run(cmd, cwd=None):
    res = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), res.stdout, res.stderr))


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle_lib(force: bool = False) -> str:
    src = os.path.join(HERE, "highreg_oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if force or not _newer(out, [src, os.path.join(HERE, "highreg_oracle.h")]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-Wall", "-Wno-unused-function",
              src, "-o", out, "-lm"])
    return out


def ref2s_lib_name(P: int, N0: int) -> str:
    return os.path.join(REF_OUT, "libref2s_P%d_N%d.so" % (P, N0))


def build_reference(force: bool = False, root: str | None = None) -> list:
    """Compile the reference programs; returns the list of built libraries.

    Does nothing (returns []) when no reference tree is found.
    """
    root = reference_root(root)
    if root is None:
        return []
    s2 = os.path.join(root, "highreg_stokes_2surf")
    e2g = os.path.join(root, "highreg_stokes_extend_to_grid")
    if not (os.path.isdir(s2) and os.path.isdir(e2g)):
        return []
    os.makedirs(REF_OUT, exist_ok=True)
    built = []
    wrap2s = os.path.join(HERE, "ref_wrap_2s.cpp")
    srcs2s = ["utilities.cpp", "surface.cpp", "stokeslets.cpp", "stresslets.cpp", "KITC.cpp", "main.cpp"]
    for P, N0 in KITC_VARIANTS:
        out = ref2s_lib_name(P, N0)
        deps = [wrap2s] + [os.path.join(s2, f) for f in srcs2s + ["KITC.h"]]
        if not force and _newer(out, deps):
            built.append(out)
            continue
        tmp = tempfile.mkdtemp(prefix="hr_ref2s_build_")
        try:
            for f in os.listdir(s2):
                if f.endswith((".cpp", ".h")):
                    shutil.copy(os.path.join(s2, f), tmp)
            kitc_h = os.path.join(tmp, "KITC.h")
            txt = open(kitc_h).read()
            txt, n1 = re.subn(r"static const int P = \d+;", "static const int P = %d;" % P, txt)
            txt, n2 = re.subn(r"static const int N0 = \d+;", "static const int N0 = %d;" % N0, txt)
            if n1 != 1 or n2 != 1:
                raise RuntimeError("KITC.h constants not found")
            open(kitc_h, "w").write(txt)
            cmd = (["g++"] + CXXFLAGS + ["-I", tmp, "-Dmain=ref2s_driver_main"]
                   + [os.path.join(tmp, f) for f in srcs2s] + [wrap2s, "-o", out])
            _run(cmd)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        built.append(out)
    out = os.path.join(REF_OUT, "librefe2g.so")
    wrape = os.path.join(HERE, "ref_wrap_e2g.cpp")
    srcse = ["utilities.cpp", "surface.cpp", "stokes.cpp", "main.cpp"]
    deps = [wrape, os.path.join(HERE, "fftw_standin", "fftw3.h")] + [os.path.join(e2g, f) for f in srcse]
    if force or not _newer(out, deps):
        cmd = (["g++"] + CXXFLAGS + ["-I", e2g, "-I", os.path.join(HERE, "fftw_standin"),
                                     "-Dmain=refe2g_driver_main"]
               + [os.path.join(e2g, f) for f in srcse] + [wrape, "-o", out])
        _run(cmd)
    built.append(out)
    return built


def build_relinked_reference(force: bool = False, root: str | None = None):
    """The reference's unmodified two-surface driver (main.cpp, surface.cpp,
    utilities.cpp) linked against the product's reference-signature layer
    (libhighreg_refapi.so) instead of its own KITC.cpp / stokeslets.cpp /
    stresslets.cpp: the drop-in test of the C++ boundary. Needs the reference
    tree and the built product library; returns the binary path or None."""
    root = reference_root(root)
    if root is None:
        return None
    s2 = os.path.join(root, "highreg_stokes_2surf")
    pkg = os.path.join(os.path.dirname(HERE), "high-order-regularization_b200")
    lib = os.path.join(pkg, "libhighreg_refapi.so")
    if not os.path.isdir(s2) or not os.path.exists(lib):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "ref2s_main_relinked")
    srcs = [os.path.join(s2, f) for f in ("main.cpp", "surface.cpp", "utilities.cpp")]
    if force or not _newer(out, srcs + [lib]):
        _run(["g++", "-std=c++14", "-O2", "-fopenmp", "-w", "-I", s2] + srcs
             + ["-o", out, "-L", pkg, "-lhighreg_refapi", "-lhighreg_b200", "-Wl,-rpath," + pkg,
                "-Wl,-rpath,$ORIGIN/../../high-order-regularization_b200"])
    return out


def build_relinked_e2g(force: bool = False, root: str | None = None):
    """The reference's unmodified extend-to-grid driver (main.cpp, stokes.cpp,
    surface.cpp, utilities.cpp: its own CPU boundary sums) compiled against
    the product's FFTW-API header and linked against libhighreg_fftw.so
    instead of FFTW, so that its Poisson solves (fftw_DST_Poisson3d_FD) run
    their transforms on the B200: the drop-in test of the Poisson boundary.
    Needs the reference tree and the built product libraries; returns the
    binary path or None."""
    root = reference_root(root)
    if root is None:
        return None
    e2g = os.path.join(root, "highreg_stokes_extend_to_grid")
    repo = os.path.dirname(HERE)
    pkg = os.path.join(repo, "high-order-regularization_b200")
    lib = os.path.join(pkg, "libhighreg_fftw.so")
    if not os.path.isdir(e2g) or not os.path.exists(lib):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "refe2g_main_relinked")
    srcs = [os.path.join(e2g, f) for f in ("main.cpp", "stokes.cpp", "surface.cpp", "utilities.cpp")]
    if force or not _newer(out, srcs + [lib]):
        _run(["g++", "-std=c++14", "-O2", "-fopenmp", "-w", "-I", e2g,
              "-I", os.path.join(repo, "include", "fftw_shim")] + srcs
             + ["-o", out, "-L", pkg, "-lhighreg_fftw", "-lhighreg_b200", "-Wl,-rpath," + pkg,
                "-Wl,-rpath,$ORIGIN/../../high-order-regularization_b200"])
    return out


def build_all(force: bool = False) -> None:
    build_oracle_lib(force)
    build_reference(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("oracle built:", os.listdir(HERE), os.listdir(REF_OUT) if os.path.isdir(REF_OUT) else [])
