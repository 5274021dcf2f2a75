"""The C-ABI library loads and exports every entry point include/jxr_b200.h
declares (no GPU needed: nothing here launches work)."""
import re
from pathlib import Path

import pytest

import jxr_b200 as J
from jxr_b200 import api

ROOT = Path(__file__).resolve().parents[1]


def declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jxrb_\w+)\s*\(", text)))


def test_every_header_function_is_exported():
    lib = J.lib()
    names = declared(ROOT / "include" / "jxr_b200.h")
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each
    assert not [n for n in names if n not in api.EXPORTS]


def test_generator_library_is_separate():
    # the generator's entry points live in their own library, not the engine's
    names = declared(ROOT / "jxr_b200" / "csrc" / "synth.h")
    synth = api.synth_lib()
    assert not [n for n in names if not hasattr(synth, n)]
    assert not [n for n in names if n not in api.SYNTH_EXPORTS]
    assert not [n for n in names if hasattr(J.lib(), n)]


def test_availability_is_false_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert J.CudaDecoderSession.is_available() is False
    with pytest.raises(J.CudaError) as e:
        J.CudaDecoderSession(0)
    assert e.value.kind == "Unavailable"


def test_autotune_candidates_and_signature():
    from jxr_b200 import autotune, workloads as W
    c = autotune.candidates()
    assert len(c) == len(set(c)) == 12
    for blocks, side in c:
        assert len(blocks) == 5 and all(1 <= b <= 3 for b in blocks) and isinstance(side, bool)
    items = W.mixed_batch(count=3, seed=1, lo=64, hi=128, threads=2)
    plans = W.plans_of(items)
    assert autotune.signature(plans) == autotune.signature(W.plans_of(items))
    assert autotune.signature(plans) != autotune.signature(plans[:2])


def test_mixed_batch_shapes():
    from jxr_b200 import workloads as W
    items = W.mixed_batch(count=12, seed=3, lo=64, hi=256, threads=2)
    for it in items:
        w, h = it.output.crop_width, it.output.crop_height
        assert 64 <= w <= 256 and 64 <= h <= 256 and w % 16 == 0 and h % 16 == 0
        assert it.kind in ("rgb420", "gray16", "rgba")
