"""bench.py's variant routing on the CPU: each variant name maps to its
storage format, streaming scheme, flow state, option flags, kernel name and
committed ncu traffic figure. No GPU is used."""
import os
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_variants_route_to_storage_streaming_and_kernel():
    from flowcraft_b200 import Storage, Streaming
    want = {
        "fp16_learned": (Storage.FP16_OFFSET, Streaming.PINGPONG, "k_bulk_pairs_learned"),
        "fp16_offset": (Storage.FP16_OFFSET, Streaming.PINGPONG, "k_bulk_pairs"),
        "fp32": (Storage.FP32, Streaming.PINGPONG, "k_bulk_pairs"),
        "fp16_aa": (Storage.FP16_OFFSET, Streaming.AA, "k_bulk_pairs_aa"),
        "fp32_aa": (Storage.FP32, Streaming.AA, "k_bulk_pairs_aa"),
        "fp16_aa_learned": (Storage.FP16_OFFSET, Streaming.AA, "k_bulk_pairs_aa_learned"),
        "fp16_tc_learned": (Storage.FP16_OFFSET, Streaming.PINGPONG, "k_bulk_pairs_learned_tc"),
        "fp16_tma": (Storage.FP16_OFFSET, Streaming.PINGPONG, "k_bulk_pairs"),
    }
    for v, (st, sm, kern) in want.items():
        assert bench.storage_of(v) == st, v
        assert bench.streaming_of(v) == sm, v
        assert bench.kernel_of(v) == f"{kern}<19,{v}>", v
        assert v in bench.BYTES_PER_ELEM, v


def test_default_variants_are_known_and_headline_is_learned():
    args = bench.parse_args([])
    variants = args.variants.split(",")
    assert variants[0] == "fp16_learned"
    for v in variants:
        bench.storage_of(v)
        assert v in bench.BYTES_PER_ELEM
    assert args.spinup > 0 and args.warmup >= 3


def test_spinup_applies_to_learned_variants_only():
    args = bench.parse_args(["--spinup", "123"])
    assert bench.spinup_of(args, "fp16_learned") == 123
    assert bench.spinup_of(args, "fp16_aa_learned") == 123
    assert bench.spinup_of(args, "fp16_offset") == 0
    assert bench.spinup_of(args, "fp32_aa") == 0


def test_bytes_per_cell_update():
    for v, elem in bench.BYTES_PER_ELEM.items():
        per_cell = 19 * 2 * elem + bench.EXTRA_BYTES.get(v, 0)
        assert per_cell == (152 if elem == 4 else 76) + (1 if v.endswith("_learned") else 0), v


def test_committed_traffic_figures_are_read():
    early = bench.ncu_traffic_per_cell("fp16_learned")
    developed = bench.ncu_traffic_per_cell("fp16_learned", developed=True)
    plain = bench.ncu_traffic_per_cell("fp16_offset")
    assert early and developed and plain
    for t in (early, developed, plain):
        assert 70.0 < t < 80.0  # about the 76-77 algorithmic bytes per cell


def test_batch_shape_option_and_candidate_table():
    """--batch-shape parses, and the Python candidate list matches the C
    header's count and the library's table (persistent shapes, one block per
    tile, then rows 0)."""
    import re
    from flowcraft_b200.batch import CANDIDATES
    assert bench.parse_args(["--batch-shape", "0x1"]).batch_shape == "0x1"
    assert bench.parse_args([]).batch_shape is None
    hdr = open(os.path.join(ROOT, "include", "fc_lbm.h")).read()
    n = int(re.search(r"#define FC_LBM_BATCH_CANDIDATES (\d+)", hdr).group(1))
    assert len(CANDIDATES) == n
    src = open(os.path.join(ROOT, "flowcraft_b200", "csrc", "fc_lbm.cu")).read()
    table = re.search(r"kBatchCand\[FC_LBM_BATCH_CANDIDATES\]\[2\] = \{(.*?)\};", src, re.S).group(1)
    pairs = [tuple(int(v) for v in m) for m in re.findall(r"\{(\d+), (\d+)\}", table)]
    assert pairs == CANDIDATES


def test_both_arms_share_the_workload_config():
    """The reference arm prints the same `config` as this arm's line (the
    driver compares them); run-dependent values stay out of it."""
    import inspect
    args = bench.parse_args([])
    cfg = bench.CONFIGS["large"]
    c = bench.workload_config(args, cfg, 1)
    assert c == bench.workload_config(args, cfg, 1)
    assert c["storage"] == args.variants.split(",")[0] and c["cells"] == cfg["nx"] * cfg["ny"] * cfg["nz"]
    assert not {"boundary_cells", "bouzidi_links", "closure_coverage", "sample_cells"} & set(c)
    for arm in (bench.run_reference_arm, bench.run_ours):
        assert "workload_config(args, cfg, world)" in inspect.getsource(arm)
