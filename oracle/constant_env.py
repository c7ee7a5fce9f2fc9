"""Test infrastructure, not product code: writes patched copies of pine's light.h and
light.cpp that add a `Constant{ color }` environment light, for the oracle build of pine
that renders the benchmark scenes (oracle/Makefile, target `ref-const`).

Pine's environment lights are the closed set {Atmosphere, Sky} (src/core/light.h:136,
factory src/core/light.cpp:158-168), so the benchmark scenes' uniform sky cannot be
expressed in pine unmodified.  The added type follows pine's own `Sky` for the part of the
sky that is not its sun (light.cpp:65-79): `Color` is the constant radiance, `Pdf` is 0, so
a path that escapes gathers it in full, and it has nothing for next-event estimation to
sample: `Sample` returns a delta sample of zero radiance at distance 0, whose shadow ray
has zero length and whose contribution is exactly 0 (RayIntegrator::EstimateDirect,
integrator.cpp:88-119).  That estimator is unbiased, and its expectation is the same as
that of the GPU renderer's constant environment, which does sample it for next-event
estimation; pine's paths simply skip that work.

Usage:  python constant_env.py <pine source root> <output src root>
Writes <out>/core/light.h and <out>/core/light.cpp; every other file comes unmodified
from the pine tree (the patched copies shadow the originals through the include order).
"""

from __future__ import annotations

import os
import sys

ADDED_TYPE = """
// Added by the oracle build (not part of pine): a uniform environment of radiance
// `color`.  Like the gradient sky of Sky it is gathered where a path escapes (Pdf 0); it
// offers next-event estimation nothing to sample (a zero-radiance delta sample).
struct ConstantEnvironment {
    static ConstantEnvironment Create(const Parameters& params);
    explicit ConstantEnvironment(Spectrum color) : color(color) {
    }

    LightSample Sample(vec3, vec2) const {
        LightSample ls;
        ls.wo = vec3(0.0f, 0.0f, 1.0f);
        ls.distance = 0.0f;
        ls.pdf = 1.0f;
        ls.Le = Spectrum(0.0f);
        ls.isDelta = true;
        return ls;
    }
    Spectrum Color(vec3) const {
        return color;
    }
    float Pdf(vec3) const {
        return 0.0f;
    }
    LightLeSample SampleLe(vec2, vec2) const {
        return {};
    }
    SpatialPdf PdfLe(const Ray&) const {
        return {};
    }
    Spectrum Power() const {
        return {};
    }
    bool IsDelta() const {
        return false;
    }

    Spectrum color;
};

"""

ADDED_CREATE = """
ConstantEnvironment ConstantEnvironment::Create(const Parameters& params) {
    return ConstantEnvironment(params.GetVec3("color"));
}
"""


def patch(src_root: str, out_root: str) -> None:
    with open(os.path.join(src_root, "core", "light.h")) as f:
        h = f.read()
    with open(os.path.join(src_root, "core", "light.cpp")) as f:
        c = f.read()
    anchor = "struct EnvironmentLight : TaggedVariant<Atmosphere, Sky> {"
    if h.count(anchor) != 1:
        raise SystemExit("light.h: the EnvironmentLight declaration was not found once")
    h = h.replace(anchor, ADDED_TYPE.lstrip("\n") +
                  "struct EnvironmentLight : TaggedVariant<Atmosphere, Sky, ConstantEnvironment> {")
    case = '        CASE("Sky") return Sky(Sky::Create(params));\n'
    if c.count(case) != 1:
        raise SystemExit("light.cpp: the Sky factory case was not found once")
    c = c.replace(case, case + '        CASE("Constant") return ConstantEnvironment('
                               'ConstantEnvironment::Create(params));\n')
    fn = "EnvironmentLight EnvironmentLight::Create("
    if c.count(fn) != 1:
        raise SystemExit("light.cpp: EnvironmentLight::Create was not found once")
    c = c.replace(fn, ADDED_CREATE.lstrip("\n") + "\n" + fn)
    os.makedirs(os.path.join(out_root, "core"), exist_ok=True)
    for name, text in (("light.h", h), ("light.cpp", c)):
        tmp = os.path.join(out_root, "core", name + ".tmp")
        with open(tmp, "w") as f:
            f.write(text)
        os.replace(tmp, os.path.join(out_root, "core", name))


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    patch(sys.argv[1], sys.argv[2])
