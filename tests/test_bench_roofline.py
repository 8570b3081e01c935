"""bench.py's roofline arithmetic on the CPU: the algorithmic byte models of
the assembly and the persistent CG at the headline size (256^2 with bending:
65,536 vertices, 130,050 triangles, 194,565 springs, 845,836 blocks), the
captured DRAM traffic's scaling with the iteration count, and the summary
object that repeats the sections' headline figures."""
import bench

INFO = {"vertices": 65536, "triangles": 130050, "springs": 194565, "blocks": 845836}


def test_assembly_bytes_model():
    # A (36 B a block), per vertex x, v, f_ext, mass, type and b, the
    # triangles' and springs' data, 8 B an incidence entry (3 a triangle, 2 a spring)
    n, t, s, b = INFO["vertices"], INFO["triangles"], INFO["springs"], INFO["blocks"]
    want = 36 * b + 77 * n + 40 * t + 24 * s + 8 * (3 * t + 2 * s)
    assert bench.algorithmic_bytes(INFO, "assemble") == want == 51602168


def test_persistent_cg_bytes_model():
    n, b = INFO["vertices"], INFO["blocks"]
    for it in (1.0, 116.5):
        want = 40 * b + 73 * n + it * (40 * b + 128 * n)
        assert abs(bench.algorithmic_bytes(INFO, f"grid_cg:{it}") - want) < 1e-3


def test_grid_cg_traffic_scaling():
    # 256^2 stays in L2: one figure for any iteration count
    assert bench.grid_cg_traffic(256, "persistent", 10) == bench.grid_cg_traffic(256, "persistent", 200)
    # 1024^2 streams the system once at the start and once per iteration
    b10 = bench.grid_cg_traffic(1024, "fused", 10)
    b21 = bench.grid_cg_traffic(1024, "fused", 21)
    assert abs(b21 / b10 - 2.0) < 1e-12
    assert bench.grid_cg_traffic(512, "fused", 10) is None


def test_summary_repeats_section_figures():
    line = {"value": 5.5e7, "e2e": {"value": 4.9e7}, "roofline": {"frac": 0.69},
            "assembly": {"ms": 0.083, "frac": 0.095}, "fp64": {"rel_dv_error": 7e-3},
            "batched": {"vertex_steps_per_s": 2.3e8, "speedup_vs_plain": 7.3, "roofline": {"frac": 0.58}},
            "serving": None, "stiff1024": None, "softbody": None}
    s = bench.summary(line)
    assert s["headline_vertex_steps_per_s"] == 5.5e7 and s["headline_e2e"] == 4.9e7
    assert s["assembly_ms"] == 0.083 and s["assembly_frac"] == 0.095
    assert s["batched_speedup_vs_plain"] == 7.3 and s["serving_vertex_steps_per_s"] is None
