"""Shader-node graphs: the scene loader compiles pine's node syntax into postfix programs
(pg_node_op), and the evaluator the kernels run (its host copy, through pg_eval_nodes and
pg_bump_normal) is compared with pine's own EvalFloat/EvalVec3 and BumpNormal on the same
inputs (tests/golden/nodes.npz, written by tests/golden/make_golden.py from the reference
built on the CPU)."""
import numpy as np
import pytest

from conftest import golden

Z = golden("nodes.npz")


def _material_scene(tmp_path, graphs, bump=None):
    """A scene with one Conductor material per graph: albedo (vec3 evaluation) and
    roughness (float evaluation) both set to the graph."""
    lines = ["Integrator: Path{\n maxDepth: 2\n sampler: Uniform{\n samplesPerPixel: 1\n }\n}",
             "Camera: ThinLen{\n film{\n size: 4 4\n }\n from: 0 0 5\n to: 0 0 0\n fov: 0.5\n}",
             "Environment: Sky{\n color: 1\n}"]
    for k, g in enumerate(graphs):
        lines.append(f"Material m{k}: Layered{{\n layer0: Conductor{{\n albedo: {g}\n"
                     f" roughness: {g}\n eta: 1.5\n }}\n}}")
        lines.append(f"Shape: Sphere{{\n position: {k} 0 0\n radius: 0.25\n material: m{k}\n}}")
    if bump is not None:
        lines.append(f"Material bumpy: Layered{{\n layer0: Diffuse{{\n albedo: 0.95\n }}\n"
                     f" bumpMap: {bump}\n}}")
        lines.append("Shape: Sphere{\n position: 0 2 0\n radius: 0.25\n material: bumpy\n}")
    path = tmp_path / "nodes.txt"
    path.write_text("\n".join(lines) + "\n")
    return str(path)


def _node_refs(desc, k):
    layer = desc.materials[k].layers[0]
    return layer.albedo_node, layer.roughness_node


@pytest.fixture(scope="module")
def parsed(tmp_path_factory):
    import pine_b200 as pb
    path = _material_scene(tmp_path_factory.mktemp("nodes"), list(Z["graphs"]),
                           bump=str(Z["bump_graph"]))
    scene = pb.ParsedScene(path)
    yield scene
    scene.close()


@pytest.mark.parametrize("k", range(len(Z["graphs"])))
def test_graph_matches_pine_both_modes(pglib, parsed, k):
    import pine_b200 as pb
    desc = parsed.desc
    vec_ref, float_ref = _node_refs(desc, k)
    assert vec_ref > 0, "every golden graph compiles to a vec3 program"
    x = Z["inputs"]
    got_vec = pb.eval_nodes(desc, vec_ref, x, "pine")
    if float_ref > 0:
        got_float = pb.eval_nodes(desc, float_ref, x, "pine")[:, 0]
    else:  # folded to a constant (Composite has no float value: node.h EvalFloat)
        got_float = np.full(len(x), desc.materials[k].layers[0].roughness, np.float32)
    want_vec, want_float = Z["vec3_out"][k], Z["float_out"][k]
    # pine mode restates pstd's sin/cos/tan/pow/sqrt and the double-precision Perlin
    # interpolation; the remaining differences are float contraction (fma) choices.
    np.testing.assert_allclose(got_vec, want_vec, rtol=2e-5, atol=2e-6, err_msg=Z["graphs"][k])
    np.testing.assert_allclose(got_float, want_float, rtol=2e-5, atol=2e-6,
                               err_msg=Z["graphs"][k])
    # Fast mode (CUDA's own functions on the device, the C library's here) stays close;
    # pstd::pow itself is an approximation good to about 1e-2 relative.
    fast = pb.eval_nodes(desc, vec_ref, x, "fast")
    np.testing.assert_allclose(fast, want_vec, rtol=1.5e-2, atol=1e-4)


def test_bump_normal_matches_pine(pglib, parsed):
    import pine_b200 as pb
    desc = parsed.desc
    ref = desc.materials[len(Z["graphs"])].bump_node
    assert ref > 0
    got = pb.bump_normal(desc, ref, Z["bump_inputs"], "pine")
    want = Z["bump_out"]
    np.testing.assert_allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-5)
    # Finite differences with delta 0.01 of a noise field: the ulp-level differences of
    # the evaluated heights are divided by 0.01, hence the looser bound than the values.
    np.testing.assert_allclose(got, want, atol=5e-4)


def test_constant_inputs_stay_constants(pglib, tmp_path):
    import pine_b200 as pb
    path = _material_scene(tmp_path, ["0.4 0.5 0.6"])
    scene = pb.ParsedScene(path)
    try:
        layer = scene.desc.materials[0].layers[0]
        assert layer.albedo_node == 0 and layer.roughness_node == 0
        assert list(layer.albedo) == pytest.approx([0.4, 0.5, 0.6])
        # pstd::stof reads the whole "0.4 0.5 0.6" as one number; the reference's node
        # harness gives the same float for this literal.
        assert layer.roughness == pytest.approx(0.23983397, rel=1e-6)
        assert scene.desc.materials[0].bump_node == 0
    finally:
        scene.close()


def test_bad_program_reference_is_rejected(pglib, parsed):
    import pine_b200 as pb
    desc = parsed.desc
    x = Z["inputs"][:4]
    for ref in (0, -1, desc.num_node_ops + 1):
        with pytest.raises(pb.PgError):
            pb.eval_nodes(desc, ref, x)
    # A reference into the middle of a program is not the start of one.
    vec_ref, _ = _node_refs(desc, 1)
    with pytest.raises(pb.PgError):
        pb.eval_nodes(desc, vec_ref + 1, x)


def test_image_texture_node_is_unsupported(pglib, tmp_path):
    import pine_b200 as pb
    path = _material_scene(tmp_path, ["Texture{\n filename: wood.png\n }"])
    with pytest.raises(pb.PgError) as e:
        pb.ParsedScene(path)
    assert e.value.status == 5  # PG_ERR_UNSUPPORTED
