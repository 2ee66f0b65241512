"""Every kernel key the bench looks up in profiles/dram_bytes_per_cell.txt
resolves to a measured DRAM figure, the table names each key once, and
every capture it cites is committed (a missing or misspelt key would leave a
bench line's roofline without its traffic)."""
import os

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLE = os.path.join(ROOT, "profiles", "dram_bytes_per_cell.txt")

# the keys bench.py passes to kernel_stats / roofline_entry
KEYS = [
    "step2_char_kernel_fp64_fma", "step2_kernel_fp64", "step2_char_kernel_fp32",
    "sweep3p_fp64", "sweep3f_fp64_fma", "sweep3f_fp32",
    "step2_char_kernel_fp64_fma_trans1", "step2_char_kernel_fp64_fma_minmod",
    "step2_char_kernel_fp64_fma_superbee", "step2_char_kernel_fp64_fma_vanleer",
    "step2_char_kernel_fp32_vanleer", "step2_char_kernel_fp64_fma_mc_vanleer",
    "step2_char_kernel_fp64_fma_runtime",
    "split3_fp64", "split2_kernel_fp64", "step2s_char_kernel_fp64_fma",
    "split2_kernel_fp64_strang", "step2s_char_kernel_fp64_fma_strang",
    "step2_kernel_euler_fp64", "step2_kernel_euler_fp64_fma",
    "step2_batch_kernel_euler", "step2_batch_kernel_euler_fp64_fma",
]


def _rows():
    out = []
    for line in open(TABLE):
        if line.startswith("#") or not line.strip():
            continue
        out.append(line.split())
    return out


def test_every_bench_key_has_a_measured_figure():
    for key in KEYS:
        nbytes, fp64 = bench.kernel_stats(key)
        assert nbytes is not None and nbytes > 0, key
        assert fp64 is None or fp64 > 0, key


def test_keys_are_unique_and_captures_committed():
    rows = _rows()
    names = [r[0] for r in rows]
    assert len(names) == len(set(names))
    for r in rows:
        cited = [w for w in r[3:] if w.startswith("profiles/")]
        assert cited, r[0]
        for path in cited:
            assert os.path.exists(os.path.join(ROOT, path.rstrip(";,"))), (r[0], path)


def test_headline_traffic_per_launch():
    cells = 4096 * 4096
    for prec, lo, hi in (("fp64_fma", 40, 48.5), ("fp64", 40, 70), ("fp32", 18, 24.5)):
        t = bench.traffic_per_launch(prec, cells)
        assert t is not None and lo * cells <= t <= hi * cells, prec
