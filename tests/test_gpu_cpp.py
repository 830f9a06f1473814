"""The C++ mirror (include/htcuda.hpp) end to end: the example program renders a serialized
scene file and its RGBA8 output equals the Python pipeline's, byte for byte."""
import os
import subprocess

import numpy as np
import pytest
import torch

from hypertrace_b200 import processing as P
from hypertrace_b200 import scene as S

pytestmark = pytest.mark.gpu
EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "hypertrace_b200", "render_scene")


@pytest.mark.parametrize("cfg", ["config0", "config1"])
def test_cpp_pipeline_matches_python(built, tmp_path, cfg):
    wl = getattr(S, cfg)()
    W, H, passes = 160, 90, 3
    scene_file = tmp_path / "scene.bin"
    scene_file.write_bytes(wl.scene.to_bytes())
    seeds = S.pixel_seeds(wl.global_seed, W * H)
    seeds_file = tmp_path / "seeds.u32"
    seeds_file.write_bytes(seeds.tobytes())
    out_file = tmp_path / "out.rgba"
    subprocess.run([EXE, str(scene_file), str(wl.scene.recipe), str(wl.scene.hops), str(W), str(H), str(passes),
                    str(seeds_file), str(out_file)], check=True, timeout=120)
    cpp = np.frombuffer(out_file.read_bytes(), dtype=np.uint8).reshape(H, W, 4)
    ctx = P.Context(0)
    pipe = P.Pipeline(ctx, (W, H), wl.scene, global_seed=wl.global_seed)
    pipe.render(passes)
    py = pipe.get_image()
    assert np.array_equal(cpp, py)


def test_cpp_reports_errors(built, tmp_path):
    (tmp_path / "scene.bin").write_bytes(b"\0" * 16)
    (tmp_path / "seeds.u32").write_bytes(b"\0" * 16)
    r = subprocess.run([EXE, str(tmp_path / "scene.bin"), "1", "4", "2", "2", "1", str(tmp_path / "seeds.u32"),
                        str(tmp_path / "o")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "htcuda error" in r.stderr
