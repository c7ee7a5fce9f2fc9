"""pine's Halton and Sobol samplers and film filters on the host: the code the kernels run
(through pg_halton_sample, pg_sobol_sample and pg_filter_table) against values pine itself
produced (tests/golden/sampler_filter.npz and sobol.npz, written by
tests/golden/make_golden.py), and the scene loader's reading of sampler and filter blocks."""
import numpy as np
import pytest

from conftest import golden

Z = golden("sampler_filter.npz")


@pytest.mark.parametrize("case", range(len(Z["halton_meta"])))
def test_halton_is_bit_exact_with_pine(pglib, case):
    import pine_b200 as pb
    w, h, scramble = (int(v) for v in Z["halton_meta"][case])
    rows = Z["halton_rows"][case]
    got = pb.halton_sample(w, h, rows, scramble=bool(scramble))
    want = Z["halton_values"][case]
    bad = got.view(np.uint32) != want.view(np.uint32)
    assert not bad.any(), f"{bad.sum()} of {len(rows)} differ, first rows {rows[bad][:4]}"


def test_halton_rejects_bad_rows(pglib):
    import pine_b200 as pb
    for row in ([0, 0, 0, 1000], [0, 0, -1, 2], [0, 0, 0, 1]):
        with pytest.raises(pb.PgError):
            pb.halton_sample(8, 8, np.array([row]))


S = golden("sobol.npz")


@pytest.mark.parametrize("case", range(len(S["meta"])))
def test_sobol_is_bit_exact_with_pine(pglib, case):
    """Sobol matrices from the Joe-Kuo direction numbers, the pixel-to-index tables derived
    from the first two dimensions, and each randomizer reproduce pine's values bit for bit."""
    import pine_b200 as pb
    w, h, k = (int(v) for v in S["meta"][case])
    rows = S["rows"][case]
    got = pb.sobol_sample(w, h, rows, randomize=str(S["strategies"][k]))
    want = S["values"][case]
    bad = got.view(np.uint32) != want.view(np.uint32)
    assert not bad.any(), f"{bad.sum()} of {len(rows)} differ, first rows {rows[bad][:4]}"


def test_sobol_rejects_bad_rows(pglib):
    import pine_b200 as pb
    for row in ([0, 0, 0, 1024], [0, 0, -1, 2], [0, 0, 0, 1], [8, 0, 0, 2]):
        with pytest.raises(pb.PgError):
            pb.sobol_sample(8, 8, np.array([row]))


def _filter_args(block):
    """(kind, radius, params) as the scene loader reads them from a film filter block."""
    kind, radius, params = "LanczosSinc", (0.5, 0.5), [3.0, 0.0]
    if block:
        kind = block.split(":")[1].split("{")[0].strip()
        fields = dict(line.strip().split(":") for line in block.splitlines()[1:-1])
        if "radius" in fields:
            r = [float(v) for v in fields["radius"].split()]
            radius = (r[0], r[1] if len(r) > 1 else r[0])
        params = {"Box": [0, 0], "Triangle": [0, 0],
                  "Gaussian": [float(fields.get("alpha", 1.0)), 0],
                  "Mitchell": [float(fields.get("B", 1 / 3)), float(fields.get("C", 1 / 3))],
                  "LanczosSinc": [float(fields.get("tau", 3.0)), 0]}[kind]
    return kind, radius, params


@pytest.mark.parametrize("k", range(len(Z["filter_blocks"])))
def test_filter_table_matches_pine(pglib, k):
    import pine_b200 as pb
    kind, radius, params = _filter_args(str(Z["filter_blocks"][k]))
    want = Z["filter_tables"][k]
    np.testing.assert_array_equal(np.float32(radius), want[:2])
    got = pb.filter_table(kind, radius, params)
    # pine's pstd::sin/exp restated; its -ffast-math build rounds trig and reassociates
    # the Mitchell polynomial, a few ulps of the table's largest value.
    np.testing.assert_allclose(got.ravel(), want[2:], rtol=1e-5,
                               atol=2e-5 * np.abs(want[2:]).max(),
                               err_msg=str(Z["filter_blocks"][k]))


def _scene(tmp_path, sampler, film_extra):
    p = tmp_path / "s.txt"
    p.write_text("Integrator: Path{\n maxDepth: 3\n sampler: " + sampler + "\n}\n"
                 "Camera: ThinLen{\n film{\n size: 16 9\n " + film_extra + "\n }\n"
                 " from: 0 0 -5\n to: 0 0 0\n fov: 0.7\n}\n"
                 "Shape: Sphere{\n position: 0 0 0\n radius: 1\n material: m\n}\n"
                 "Material m: Layered{\n layer0: Diffuse{\n albedo: 0.5\n }\n}\n")
    return str(p)


@pytest.mark.parametrize("sampler,kind,spp,scramble", [
    ("Halton{\n samplesPerPixel: 32\n }", 1, 32, 1),
    ("Halton{\n samplesPerPixel: 8\n randomizeStrategy: none\n }", 1, 8, 0),
    ("Uniform{\n samplesPerPixel: 5\n }", 0, 5, 1),
    ("Sobol{\n samplesPerPixel: 16\n }", 2, 16, 2),
    ("Sobol{\n samplesPerPixel: 4\n randomizeStrategy: none\n }", 2, 4, 0),
    ("Sobol{\n samplesPerPixel: 4\n randomizeStrategy: Owen\n }", 2, 4, 3),
    ("Sobol{\n samplesPerPixel: 4\n randomizeStrategy: binaryPermutate\n }", 2, 4, 1),
    ("Sobol{\n samplesPerPixel: 4\n randomizeStrategy: other\n }", 2, 4, 1),
    ("Stratified{\n xPixelSamples: 3\n yPixelSamples: 4\n }", 0, 12, 1),
    ("ZeroTwoSequence{\n samplesPerPixel: 5\n }", 0, 8, 1),
])
def test_loader_reads_samplers(pglib, tmp_path, sampler, kind, spp, scramble):
    import pine_b200 as pb
    ps = pb.ParsedScene(_scene(tmp_path, sampler, ""))
    d = ps.desc
    assert (d.sampler, d.samples_per_pixel, d.sampler_scramble) == (kind, spp, scramble)
    ps.close()


@pytest.mark.parametrize("k", range(len(Z["filter_blocks"])))
def test_loader_reads_filters(pglib, tmp_path, k):
    import pine_b200 as pb
    block = str(Z["filter_blocks"][k])
    kind, radius, params = _filter_args(block)
    ps = pb.ParsedScene(_scene(tmp_path, "Halton{\n samplesPerPixel: 1\n }", block))
    d = ps.desc
    assert d.filter == pb.FILTERS[kind]
    np.testing.assert_allclose(list(d.filter_radius), radius)
    np.testing.assert_allclose(list(d.filter_params), params, rtol=1e-6)
    ps.close()


@pytest.mark.parametrize("itype,kind", [("Path", 0), ("RandomWalk", 1), ("GpuPath", 0)])
def test_loader_reads_integrators(pglib, tmp_path, itype, kind):
    import pine_b200 as pb
    path = _scene(tmp_path, "Uniform{\n samplesPerPixel: 2\n }", "")
    with open(path) as f:
        text = f.read().replace("Integrator: Path{", "Integrator: " + itype + "{")
    with open(path, "w") as f:
        f.write(text)
    ps = pb.ParsedScene(path)
    assert ps.desc.integrator == kind
    ps.close()
