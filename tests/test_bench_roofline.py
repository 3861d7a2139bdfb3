"""The bench line's roofline bookkeeping, on the CPU: the algorithmic bytes follow each form's stencil precision, every
group with a recorded DRAM traffic has a binding, and the traffic scales with the workload's level-0 pixels."""
import importlib.util
import os

import pytest

from nntc_b200 import materials

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_stencil_bytes_follow_the_form(bench):
    mat = materials.small(5, 64, 48, textures=2, c0=4, c1=4)
    t0 = sum(p[0] * p[1] for p in mat.planes)
    t1 = sum(p[2] * p[3] for p in mat.planes)
    # the CG product reads 5 blocks of C x C coefficients per texel: 8 bytes each in the plain form, 4 in the adjoint
    d = bench.algorithmic_bytes("cg_product_level0", mat, "plain") - bench.algorithmic_bytes("cg_product_level0", mat,
                                                                                             "adjoint")
    assert d == t0 * 5 * 16 * 4
    d1 = bench.algorithmic_bytes("cg_product_level1", mat, "plain") - bench.algorithmic_bytes("cg_product_level1", mat,
                                                                                              "adjoint")
    assert d1 == t1 * 5 * 16 * 4
    # the BC refine reads the FP64 stencil in both forms
    assert bench.algorithmic_bytes("bc_refine", mat, "plain") == bench.algorithmic_bytes("bc_refine", mat, "adjoint")


def test_traffic_groups_have_bindings(bench):
    for form, groups in bench.TRAFFIC_PER_UNIT.items():
        for name, per_pixel in groups.items():
            assert per_pixel > 0
            assert bench.BINDING[form].get(name), (form, name)


def test_roofline_scales_traffic_by_level0_pixels(bench):
    mat = materials.small(7, 96, 64, textures=2, c0=4, c1=4)
    t0 = sum(p[0] * p[1] for p in mat.planes)
    roof = bench.roofline("bc_refine", (4, 8.0), mat, 6000.0, 1500.0, "fallback", "adjoint")
    assert roof["traffic"] == round(bench.TRAFFIC_PER_UNIT["adjoint"]["bc_refine"] * t0)
    assert roof["ms_per_launch"] == 2.0
    per = bench.algorithmic_bytes("bc_refine", mat, "adjoint")
    assert abs(roof["achieved"] - round(per / 0.002 / 1e9, 2)) < 1e-6
    assert roof["binding"] == bench.BINDING["adjoint"]["bc_refine"]
