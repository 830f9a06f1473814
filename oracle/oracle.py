"""ctypes front end of the CPU oracles. TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:
  * libhtoracle_f32.so / libhtoracle_f64.so  -- the C restatement (htoracle.c);
  * _ref/libhtref_f32.so / _ref/libhtref_f64.so -- the reference's own kernel sources
    compiled as host C++ (ref/Makefile), present where the reference tree was available
    when the repository was built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module;
the product (hypertrace_b200) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

JITTER_YX = 1  # first jitter draw -> y, as the g++-compiled reference evaluates random_uniform2

_libs = {}


def build(reference_root: Optional[str] = None) -> None:
    """Compile the restatement (always) and oracle/_ref from the reference tree at
    `reference_root` (or $HT_REFERENCE_ROOT) when one is given and present."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = reference_root or os.environ.get("HT_REFERENCE_ROOT")
    if ref and os.path.isdir(os.path.join(ref, "kernel", "ocl")):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF={ref}"], check=True)


def _load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run oracle.build())")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def ref_available(precision: int = 32) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libhtref_f{precision}.so"))


_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_f32p = ctypes.POINTER(ctypes.c_float)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class RenderResult:
    def __init__(self, canvas: np.ndarray, seeds: np.ndarray, stats: np.ndarray):
        self.canvas = canvas
        self.seeds = seeds
        self.stats = {"samples": int(stats[0]), "hops": int(stats[1]),
                      "object_tests": int(stats[2]), "hits": int(stats[3])}


def render(scene_bytes: bytes, recipe: int, hops: int, width: int, height: int,
           pixels: Sequence[int], seeds: np.ndarray, passes: int = 1,
           canvas: Optional[np.ndarray] = None, precision: int = 32, flags: int = 0,
           threads: int = 1, address_width: int = 32, impl: str = "port") -> RenderResult:
    """Render `passes` passes over `pixels` (indices into a width x height image).

    impl="port" uses the C restatement, impl="reference" the reference's compiled kernel
    (which always uses the g++ jitter order, i.e. flags must contain JITTER_YX to compare).
    """
    pix = np.ascontiguousarray(np.asarray(pixels, dtype=np.uint32))
    n = pix.shape[0]
    sd = np.array(seeds, dtype=np.uint32, copy=True)
    if sd.shape != (n,):
        raise ValueError("seeds must have one entry per listed pixel")
    cv = np.zeros((n, 4), dtype=np.float32) if canvas is None else np.array(canvas, dtype=np.float32, copy=True)
    st = np.zeros(4, dtype=np.uint64)
    buf = np.frombuffer(scene_bytes, dtype=np.uint8)
    if impl == "port":
        lib = _load(os.path.join(HERE, f"libhtoracle_f{precision}.so"))
        fn = getattr(lib, f"hto{precision}_render")
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_int, ctypes.c_uint32, _u8p, ctypes.c_size_t, ctypes.c_int,
                       ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.c_size_t, ctypes.c_uint32,
                       _f32p, _u32p, ctypes.c_uint32, ctypes.c_int, _u64p]
        rc = fn(recipe, hops, _ptr(buf, _u8p), len(scene_bytes), address_width, width, height,
                _ptr(pix, _u32p), n, passes, _ptr(cv, _f32p), _ptr(sd, _u32p), flags, threads,
                _ptr(st, _u64p))
    elif impl == "reference":
        if address_width != 32:
            raise ValueError("the reference harness parses X32 scenes")
        lib = _load(os.path.join(REF_DIR, f"libhtref_f{precision}.so"))
        fn = lib.htref_render if recipe in (1, 2) else lib.htref_render_ext
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_int, ctypes.c_uint32, _u8p, ctypes.c_size_t, ctypes.c_uint32,
                       ctypes.c_uint32, _u32p, ctypes.c_size_t, ctypes.c_uint32, _f32p, _u32p,
                       ctypes.c_int, _u64p]
        rc = fn(recipe, hops, _ptr(buf, _u8p), len(scene_bytes), width, height, _ptr(pix, _u32p),
                n, passes, _ptr(cv, _f32p), _ptr(sd, _u32p), threads, _ptr(st, _u64p))
    else:
        raise ValueError(impl)
    if rc != 0:
        raise RuntimeError(f"oracle render failed with status {rc}")
    return RenderResult(cv, sd, st)


def extract_gamma_pack(canvas: np.ndarray, passes: int, gamma: float):
    """Post chain on the CPU: returns (float image, packed RGBA8)."""
    lib = _load(os.path.join(HERE, "libhtoracle_f32.so"))
    fn = lib.hto32_extract_gamma_pack
    fn.restype = None
    fn.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, _f32p, _f32p, _u8p]
    cv = np.ascontiguousarray(canvas, dtype=np.float32).reshape(-1, 4)
    img = np.zeros_like(cv)
    packed = np.zeros(cv.shape, dtype=np.uint8)
    fn(cv.shape[0], passes, gamma, _ptr(cv, _f32p), _ptr(img, _f32p), _ptr(packed, _u8p))
    return img, packed


def pack(image: np.ndarray) -> np.ndarray:
    """Pack alone on the CPU (canvas.rs:176-186): float image -> RGBA8, toward zero."""
    lib = _load(os.path.join(HERE, "libhtoracle_f32.so"))
    fn = lib.hto32_pack
    fn.restype = None
    fn.argtypes = [ctypes.c_uint32, _f32p, _u8p]
    img = np.ascontiguousarray(image, dtype=np.float32).reshape(-1, 4)
    packed = np.zeros(img.shape, dtype=np.uint8)
    fn(img.shape[0], _ptr(img, _f32p), _ptr(packed, _u8p))
    return packed


def rng_uniforms(seed: int, n: int, impl: str = "port", precision: int = 32):
    out = np.zeros(n, dtype=np.float64)
    state = ctypes.c_uint32(0)
    if impl == "port":
        lib = _load(os.path.join(HERE, f"libhtoracle_f{precision}.so"))
        fn = getattr(lib, f"hto{precision}_rng_uniforms")
    else:
        lib = _load(os.path.join(REF_DIR, f"libhtref_f{precision}.so"))
        fn = lib.htref_rng_uniforms
    fn.restype = None
    fn.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double), _u32p]
    fn(seed, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(state))
    return out, state.value
