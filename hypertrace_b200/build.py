"""Build libhtcuda.so in-tree for sm_100a.

    python -m hypertrace_b200.build

Flags: FMA contraction off (-fmad=false) and IEEE division / square root (the nvcc
defaults without --use_fast_math) so the float path rounds exactly like the reference's
kernel library compiled for the host.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRCS = [os.path.join(HERE, "csrc", "htcuda.cu"), os.path.join(HERE, "csrc", "htgeneric.cu"),
        os.path.join(HERE, "csrc", "htserve.cu")]
OUT = os.path.join(HERE, "libhtcuda.so")
# Device headers that htc_program_build hands to NVRTC, embedded as C strings.
NVRTC_HEADERS = [("k_header_ht_math", "ht_math.cuh"), ("k_header_ht_bound", "ht_bound.cuh"),
                 ("k_header_ht_generic", "ht_generic.cuh")]
GENERATED = os.path.join(HERE, "csrc", "generated", "nvrtc_headers.inc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared",
    "-diag-suppress", "177",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    return "nvcc"


def sources():
    csrc = os.path.join(HERE, "csrc")
    return [os.path.join(csrc, f) for f in sorted(os.listdir(csrc))
            if f.endswith((".cu", ".cuh", ".h", ".hpp"))] + [os.path.join(ROOT, "include", "htcuda.h"), GENERATED]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def c_string(text: str) -> str:
    out = []
    for line in text.splitlines(True):
        esc = line.replace("\\", "\\\\").replace('"', '\\"').replace("\n", "\\n")
        out.append('"' + esc + '"')
    return "\n".join(out) if out else '""'


def gen_headers() -> str:
    """Writes csrc/generated/nvrtc_headers.inc (the NVRTC header texts) when stale."""
    os.makedirs(os.path.dirname(GENERATED), exist_ok=True)
    parts = ["// generated by hypertrace_b200/build.py from the files named below; do not edit\n"]
    for var, name in NVRTC_HEADERS:
        with open(os.path.join(HERE, "csrc", name)) as f:
            parts.append("// %s\nstatic const char %s[] =\n%s;\n" % (name, var, c_string(f.read())))
    text = "".join(parts)
    old = open(GENERATED).read() if os.path.exists(GENERATED) else None
    if old != text:
        with open(GENERATED, "w") as f:
            f.write(text)
    return GENERATED


def build(force: bool = False, verbose: bool = False) -> str:
    gen_headers()
    if not force and up_to_date():
        return OUT
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT] + SRCS
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    return OUT


EXAMPLE_SRC = os.path.join(HERE, "csrc", "examples", "render_scene.cpp")
EXAMPLE_OUT = os.path.join(HERE, "render_scene")


def build_example(force: bool = False) -> str:
    """The C++ example over include/htcuda.hpp, linked against libhtcuda.so."""
    deps = [EXAMPLE_SRC, os.path.join(ROOT, "include", "htcuda.hpp"), os.path.join(ROOT, "include", "htcuda.h"), OUT]
    if not force and os.path.exists(EXAMPLE_OUT) and all(os.path.getmtime(d) <= os.path.getmtime(EXAMPLE_OUT) for d in deps):
        return EXAMPLE_OUT
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", EXAMPLE_SRC, "-o", EXAMPLE_OUT,
           "-L" + HERE, "-lhtcuda", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    return EXAMPLE_OUT


SELFTEST_SRC = os.path.join(ROOT, "tests", "cuda", "ht_selftest.cu")
SELFTEST_OUT = os.path.join(ROOT, "tests", "cuda", "libht_selftest.so")


def build_selftest(force: bool = False) -> str:
    """Test-only device unit tests (tests/cuda/ht_selftest.cu), same flags as the library."""
    if not os.path.exists(SELFTEST_SRC):
        return ""
    srcs = sources() + [SELFTEST_SRC]
    if not force and os.path.exists(SELFTEST_OUT) and all(os.path.getmtime(s) <= os.path.getmtime(SELFTEST_OUT) for s in srcs):
        return SELFTEST_OUT
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", SELFTEST_OUT, SELFTEST_SRC]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    return SELFTEST_OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
