"""The Python mirror of the reference's entity types (hypertrace_b200/types.py).

1. Layout: the generic layout rules (type-macros/src/entity.rs) reproduce the hand-derived
   byte ABI of the hearth / Euclidean recipes exactly (scene.serialize), for address
   widths 32 and 64, and give the object strides the reference's own instantiation
   (oracle/ref/ref_scenes_ext.cpp) and the C port assume.
2. The example scene types (main/examples/hy.rs, eu.rs): the C port reproduces the
   reference's kernel compiled for the host on random scenes of those types.
"""
import numpy as np
import pytest

from hypertrace_b200 import scene as S
from hypertrace_b200 import types as T
from oracle import oracle


@pytest.mark.parametrize("cfg", [S.config0, S.config1, S.config2])
@pytest.mark.parametrize("aw", [32, 64])
def test_generic_layout_matches_recipe_bytes(cfg, aw):
    sc = cfg().scene
    ty = T.hearth_type() if sc.recipe == S.RECIPE_HY else T.euclid_type()
    assert T.serialize(ty, T.hearth_value(sc), aw) == S.serialize(sc, aw)
    assert T.static_size(ty, aw) == (S.HY_OBJECTS_OFFSET if sc.recipe == S.RECIPE_HY else S.EU_OBJECTS_OFFSET)


@pytest.mark.parametrize("aw", [32, 64])
def test_example_type_layouts(aw):
    W = aw // 8
    hy = T.hy_tiled_type()
    obj = hy.fields[3][1].elem
    assert obj.lay(W) == (384, 32)
    assert hy.offsets(W) == [0, 0, 64, 96] and T.static_size(hy, aw) == 128
    m = T.hy_tiled_material()
    assert m.lay(W) == (64, 16)
    mix = m.fields[1][1]
    assert [o + 16 for o in mix.offsets(W)] == [16, 48, 52]
    eu = T.eu_gradient_type()
    assert eu.fields[3][1].elem.lay(W) == (128, 16)
    assert eu.offsets(W) == [0, 0, 48, 112] and T.static_size(eu, aw) == 128
    cov = eu.fields[3][1].elem.fields[2][1]
    assert [16 + o for o in cov.offsets(W)] == [16, 16, 112]
    # the 64-bit scene differs only in the high words of the usize slots
    a = T.serialize(hy, T.hy_example_value(), 32)
    b = T.serialize(hy, T.hy_example_value(), 64)
    assert len(a) == len(b)
    diff = [i for i in range(len(a)) if a[i] != b[i]]
    assert diff == []


@pytest.mark.parametrize("aw", [32, 64])
def test_compound_type_layout(aw):
    """Offsets the reference's instantiation and the C port read (oracle/ref/ref_scenes_ext.cpp):
    object map Chain<Linear3, Shift3> @128 (linear @128, shift @192), material @256, shape
    vector count @384, elements @448 + 192 i (shift @0, linear @64, choice @128)."""
    W = aw // 8
    ty = T.eu_compound_type()
    assert ty.offsets(W) == [0, 0, 48, 128] and T.static_size(ty, aw) == 448
    obj = ty.fields[3][1]
    assert obj.offsets(W) == [0, 0, 128] and obj.fields[1][1].lay(W) == (128, 64)
    cov = obj.fields[2][1]
    assert cov.offsets(W) == [0, 0, 128]
    elem = cov.fields[2][1].elem
    assert elem.lay(W) == (192, 64) and elem.offsets(W) == [0, 0, 128]
    val = T.eu_compound_random_value(1, 5)
    data = T.serialize(ty, val, aw)
    assert len(data) == 448 + 5 * 192
    lin = np.frombuffer(data[128:192], dtype=np.float32).reshape(4, 4)
    assert np.allclose(lin[:3, :3], val["object"]["map"][0], atol=1e-6) and list(lin[3]) == [0, 0, 0, 1]
    assert list(lin[:3, 3]) == [0, 0, 0]


def test_cxx_names():
    assert T.hy_tiled_type().cxx().startswith("SceneImpl<Hy, MappedView<Hy, PointView<Hy>, Moebius>, ObjectVec<Hy,")
    assert "ShapeChoice<Eu, PlaneEu, Sphere, Cube>" in T.eu_gradient_type().cxx()
    assert T.Homogenous3().cxx() == "Homogenous3"
    assert T.Chain(T.Rotation3(), T.Shift3()).cxx() == "Chain<Rotation3, Shift3>"


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [11, 22, 33])
@pytest.mark.parametrize("recipe", [3, 4, 5])
def test_port_matches_reference_example_types(built, seed, recipe):
    if recipe == 3:
        data = T.serialize(T.hy_tiled_type(), T.hy_tiled_random_value(seed, n_objects=6))
        hops = 4
    elif recipe == 5:   # the compound type: Linear3 chains, shape vector of mapped shapes
        data = T.serialize(T.eu_compound_type(), T.eu_compound_random_value(seed, 7))
        hops = 6
    else:
        data = T.serialize(T.eu_gradient_type(), T.eu_gradient_random_value(seed, n_objects=7))
        hops = 5
    W, H = 48, 36
    pix = np.arange(W * H, dtype=np.uint32)
    seeds = S.pixel_seeds(seed, W * H)
    for precision in (32, 64):
        ref = oracle.render(data, recipe, hops, W, H, pix, seeds, passes=2, impl="reference",
                            precision=precision, threads=4)
        port = oracle.render(data, recipe, hops, W, H, pix, seeds, passes=2, flags=oracle.JITTER_YX,
                             precision=precision, threads=4)
        assert np.array_equal(ref.seeds, port.seeds)
        assert np.array_equal(ref.canvas.view(np.uint32), port.canvas.view(np.uint32))
        assert ref.stats == port.stats
        assert ref.stats["hits"] > 0


def test_port_rejects_bad_variant(built):
    data = bytearray(T.serialize(T.hy_tiled_type(), T.hy_example_value()))
    data[128 + 32:128 + 36] = (9).to_bytes(4, "little")
    with pytest.raises(RuntimeError):
        oracle.render(bytes(data), 3, 3, 8, 8, [0], [1])
    data = bytearray(T.serialize(T.eu_gradient_type(), T.eu_example_value()))
    data[128 + 112:128 + 116] = (3).to_bytes(4, "little")
    with pytest.raises(RuntimeError):
        oracle.render(bytes(data), 4, 4, 8, 8, [0], [1])
