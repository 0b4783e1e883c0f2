"""Build recipe of the CPU oracles (TEST INFRASTRUCTURE ONLY).

    python oracle/build.py [--force] [--reference DIR]

1. ``oracle/lib/libmorpho_oracle.so`` -- this project's C++/OpenMP
   restatement of the reference's per-step algorithm (morpho_oracle.cpp).
2. When a reference tree is given (``--reference DIR`` or
   ``$MORPHOSHELL_REFERENCE``; DIR holds ``source_files/``) and present,
   the reference's own C++ files compiled
   unmodified with g++ against ``oracle/eigen_shim`` (Eigen 3 is not installed
   here), outputs only under ``oracle/_ref/``:
     _ref/libmorpho_ref.so     every source file except main.cpp, plus
                               ref_bridge.cpp (the ref_* C ABI of oracle.h),
                               plus do_dialling.cpp once more per dialling
                               protocol 2..5 with that protocol's block
                               switched on (edit applied in memory)
     _ref/morphoshell_ref      the reference's whole executable, as shipped
                               (dialling protocol 1)
     _ref/morphoshell_ref_p3   the same with do_dialling.cpp's protocol-3 block
                               switched on, the way the reference expects a user
                               to select a protocol (edit applied in memory,
                               piped to g++; nothing is written to the tree)
   Flags follow the reference Makefile (-O3 -fopenmp -std=c++17) with
   -march=x86-64-v3 instead of -march=native so the objects run on any
   AVX2 host they are copied to.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
REF_OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "eigen_shim")
CXX = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-w"]

PORT_LIB = os.path.join(LIB_DIR, "libmorpho_oracle.so")
REF_LIB = os.path.join(REF_OUT, "libmorpho_ref.so")
REF_EXE = os.path.join(REF_OUT, "morphoshell_ref")
REF_EXE_P3 = os.path.join(REF_OUT, "morphoshell_ref_p3")


def _run(cmd, stdin=None):
    r = subprocess.run(cmd, input=stdin, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build step failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def _newer(out, *srcs):
    return os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs)


def build_port(force=False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    src = os.path.join(HERE, "morpho_oracle.cpp")
    hdr = os.path.join(HERE, "oracle.h")
    if force or not _newer(PORT_LIB, src, hdr):
        _run(CXX + ["-shared", "-o", PORT_LIB, src])
    return PORT_LIB


def protocol_source(text: str, k: int) -> str:
    """do_dialling.cpp with protocol 1 commented out and the protocol-k
    block (k = 2..5, between the comment lines that open and close it)
    uncommented, the way the reference expects a user to select a protocol
    (do_dialling.cpp:70-73)."""
    lines = text.split("\n")
    out = []
    p1 = ("abar_comps = (1.0-dial_factor) * a_comps_at_zero_dial_factor + dial_factor * abar_info;",
          "bbar_comps = (1.0-dial_factor) * b_comps_at_zero_dial_factor + dial_factor * bbar_info;")
    marker = next(i for i, l in enumerate(lines) if l.strip() == "// %d)" % k)
    opener = max(i for i in range(marker) if lines[i].strip() == "/*")
    closer = next(i for i in range(marker, len(lines)) if lines[i].strip() == "*/")
    n_p1 = 0
    for i, l in enumerate(lines):
        if i in (opener, closer):
            continue
        if l.strip() in p1:
            out.append("// " + l)
            n_p1 += 1
            continue
        out.append(l)
    if n_p1 != 2:
        raise RuntimeError("protocol-1 lines not found in do_dialling.cpp")
    return "\n".join(out)


def protocol3_source(text: str) -> str:
    return protocol_source(text, 3)


def reference_sources(reference=None):
    """source_files/ of the reference tree named by the argument or by
    $MORPHOSHELL_REFERENCE, or None when neither names an existing tree."""
    root = reference or os.environ.get("MORPHOSHELL_REFERENCE")
    if not root:
        return None
    src = os.path.join(root, "source_files")
    return src if os.path.isdir(src) else None


def build_ref(force=False, reference=None):
    ref_src = reference_sources(reference)
    if ref_src is None:
        return None
    obj_dir = os.path.join(REF_OUT, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    shim_hdrs = [os.path.join(SHIM, "Eigen", h) for h in ("Dense", "Sparse")]
    srcs = sorted(glob.glob(os.path.join(ref_src, "*.cpp")))
    inc = ["-I" + SHIM, "-I" + ref_src]

    def comp(src):
        obj = os.path.join(obj_dir, os.path.basename(src)[:-4] + ".o")
        if force or not _newer(obj, src, *shim_hdrs):
            _run(CXX + inc + ["-c", src, "-o", obj])
        return obj

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(comp, srcs))
    dd = os.path.join(ref_src, "do_dialling.cpp")
    proto_objs = []
    for k in (2, 3, 4, 5):
        pk_obj = os.path.join(obj_dir, "do_dialling_protocol%d.o" % k)
        if force or not _newer(pk_obj, dd, *shim_hdrs):
            with open(dd) as f:
                text = protocol_source(f.read(), k)
            _run(CXX + inc + ["-Ddo_dialling=do_dialling_protocol%d" % k, "-x", "c++", "-c", "-", "-o", pk_obj],
                 stdin=text)
        proto_objs.append(pk_obj)
    p3_main_obj = os.path.join(obj_dir, "do_dialling_p3_as_default.o")
    if force or not _newer(p3_main_obj, dd, *shim_hdrs):
        with open(dd) as f:
            text = protocol3_source(f.read())
        _run(CXX + inc + ["-x", "c++", "-c", "-", "-o", p3_main_obj], stdin=text)
    bridge = os.path.join(HERE, "ref_bridge.cpp")
    bridge_obj = os.path.join(obj_dir, "ref_bridge.o")
    if force or not _newer(bridge_obj, bridge, os.path.join(HERE, "oracle.h"), *shim_hdrs):
        _run(CXX + inc + ["-c", bridge, "-o", bridge_obj])
    main_obj = os.path.join(obj_dir, "main.o")
    dd_obj = os.path.join(obj_dir, "do_dialling.o")
    lib_objs = [o for o in objs if o != main_obj] + proto_objs + [bridge_obj]
    if force or not _newer(REF_LIB, *lib_objs):
        _run(CXX + ["-shared", "-o", REF_LIB] + lib_objs)
    if force or not _newer(REF_EXE, *objs):
        _run(CXX + ["-o", REF_EXE] + objs)
    p3_objs = [o for o in objs if o != dd_obj] + [p3_main_obj]
    if force or not _newer(REF_EXE_P3, *p3_objs):
        _run(CXX + ["-o", REF_EXE_P3] + p3_objs)
    return REF_LIB


def build(force=False, reference=None):
    port = build_port(force)
    ref = build_ref(force, reference)
    return port, ref


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--reference", default=None, help="reference tree (holds source_files/)")
    a = ap.parse_args()
    print(build(a.force, a.reference))
    sys.exit(0)
