"""Tuned kernel options (edus_b200/autotune.py) as the batch and the server
take them from the tuning cache, on the CPU."""
import json

from edus_b200 import abi, autotune


def test_mixed_batches_take_fp64_tuning_for_their_fp64_classes(tmp_path, monkeypatch):
    """Mixed-precision batches run the 2- and 3-band classes in FP64, so those
    classes get the FP64 kernels' tuned tile and register profile; 4 bands and
    up keep the mixed-precision entries."""
    cache = {"GPU X": {
        "fp64": {"2": {"tile_k": 32, "regs_profile": 1}, "3": {"tile_k": 16, "regs_profile": 0},
                 "8": {"tile_k": 8, "regs_profile": 0}},
        "mixed": {"2": {"tile_k": 32, "regs_profile": 3}, "8": {"tile_k": 16, "regs_profile": 4},
                  "16": {"tile_k": 4, "regs_profile": 4}},
    }}
    path = tmp_path / "tuned.json"
    path.write_text(json.dumps(cache))
    monkeypatch.setenv("EDUS_TUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "gpu_name", lambda: "GPU X")
    tile, prof = autotune.tuned_options(abi.EDUS_PREC_MIXED)
    assert tile == {2: 32, 3: 16, 8: 16, 16: 4}
    assert prof == {2: 1, 3: 0, 8: 4, 16: 4}
    tile, prof = autotune.tuned_options(abi.EDUS_PREC_FP64)
    assert tile == {2: 32, 3: 16, 8: 8} and prof == {2: 1, 3: 0, 8: 0}


def test_untuned_gpu_gives_empty_options(tmp_path, monkeypatch):
    monkeypatch.setenv("EDUS_TUNE_CACHE", str(tmp_path / "missing.json"))
    assert autotune.tuned_options(abi.EDUS_PREC_MIXED) == ({}, {})
