"""Build recipe of the native library libtimbir_b200.so (sm_100a).

Compiles the CUDA kernels and the C/C++ host driver in timbir_b200/csrc with
nvcc into one shared library placed beside this file, exporting the C ABI of
include/mbir4d.h and include/timbir_b200.h.  Run ``python -m timbir_b200.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtimbir_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["mbir_kernels.cu", "mbir_sv.cu", "mbir_fbp.cu", "warm_net.cu", "mbir_stage.cu", "mbir_noalloc.cu", "mbir_nhicd.cu", "mbir_ingest.cu", "mbir_setup.cpp", "mbir_reconstruct.cpp"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(HERE, "..", "include", f) for f in ("mbir4d.h", "timbir_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def sources_digest() -> str:
    """SHA-256 over the library's sources and public headers, in a fixed order."""
    import hashlib
    h = hashlib.sha256()
    names = sorted(os.listdir(CSRC))
    for n in names:
        with open(os.path.join(CSRC, n), "rb") as f:
            h.update(n.encode() + b"\0" + f.read())
    for n in ("mbir4d.h", "timbir_b200.h"):
        with open(os.path.join(HERE, "..", "include", n), "rb") as f:
            h.update(n.encode() + b"\0" + f.read())
    return h.hexdigest()


INFO = os.path.join(HERE, "_build", "build_info.json")


def build_info() -> dict:
    """What the last build() did: the sources' digest the library was built
    from, and whether that call compiled or found the library current."""
    import json
    try:
        with open(INFO) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _record(compiled: bool) -> None:
    import json
    import time
    os.makedirs(os.path.dirname(INFO), exist_ok=True)
    info = build_info() if not compiled else {}
    info.update({"sources_sha256": sources_digest() if compiled else info.get("sources_sha256", sources_digest()),
                 "compiled_by_last_call": compiled, "time": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())})
    with open(INFO, "w") as f:
        json.dump(info, f)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        _record(False)
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    env = dict(os.environ)
    env.pop("CC", None)  # nvcc's host compiler is the system gcc
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "--extended-lambda", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off",
               "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
    subprocess.run(cmd, check=True, env=env)
    _record(True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
