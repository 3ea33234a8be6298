"""Launch tuning: the C ABI's tunables and the autotuner's committed choices
(host-only; no GPU needed)."""
import json
import os

import pytest

import ntt_gpu_b200 as nb

EXPECTED = {"ntt_minb_fwd_col", "ntt_minb_fwd_row", "ntt_minb_inv_row", "ntt_minb_inv_col",
            "ntt_col_direct", "ntt_row_direct", "ntt_epi_stage", "intt_unscaled", "digits_lazy", "ntt_stage_tw_fwd_row",
            "ntt_stage_tw_inv_row", "conv_limbs", "conv_blocks_per_sm", "conv_tc_tiles", "conv_tc_fixed",
            "mac_limbs", "mac_approx", "mac_rotate", "conv_tc", "row_mac", "row_mac_max_beta",
            "row_mac_inv_rows", "host_chunk_towers", "ntt_cluster"}


def test_tunables_are_listed_and_range_checked():
    names = set(nb.tuning_names())
    assert names == EXPECTED
    before = nb.tuning_get("ntt_minb_fwd_row")
    try:
        nb.tuning_set("ntt_minb_fwd_row", 3)
        assert nb.tuning_get("ntt_minb_fwd_row") == 3
        with pytest.raises(nb.ContractError):
            nb.tuning_set("ntt_minb_fwd_row", 5)
        with pytest.raises(nb.ContractError):
            nb.tuning_set("no_such_tunable", 1)
    finally:
        nb.tuning_set("ntt_minb_fwd_row", before)


def test_committed_tuning_file_is_valid_and_applied():
    if not os.path.exists(nb.TUNING):
        pytest.skip("no tuning.json committed")
    with open(nb.TUNING) as f:
        tuning = json.load(f)
    assert set(tuning["choices"]) <= EXPECTED
    for name, value in tuning["choices"].items():
        assert nb.tuning_get(name) == value  # load() applied it
        assert str(value) in tuning["measurements"][name]["device_ms_per_call"]
