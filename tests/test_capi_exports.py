"""The C-ABI library loads without a GPU and exports every entry point include/nwg_capi.h declares."""
import ctypes
import importlib
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "nwg_capi.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(nwg_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for required in ["nwg_create", "nwg_destroy", "nwg_bootstrap", "nwg_evaluate", "nwg_read_summary",
                     "nwg_advance", "nwg_swap_generations", "nwg_read_status", "nwg_status_string",
                     "nwg_download_slot", "nwg_download_current_generation", "nwg_upload_catalog"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    pkg = importlib.import_module("neuroevolutionary-wordle_b200")
    from importlib import import_module

    build = import_module("neuroevolutionary-wordle_b200.build")
    build.build()
    lib = ctypes.CDLL(str(pkg.capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pkg.capi.EXPORTS) <= set(declared_functions())


def test_status_strings_match_reference_codes():
    pkg = importlib.import_module("neuroevolutionary-wordle_b200")
    s = pkg.capi.status_string
    assert s(0) == "ok"
    assert s(6) == "could not append a model-selected guess to the Wordle grid"
    assert s(8) == "output-embedding action selection failed"
    assert s(14) == "slab is genuinely full"
    assert s(99) == "unknown slab ga runtime status"


def test_abi_version():
    pkg = importlib.import_module("neuroevolutionary-wordle_b200")
    assert pkg.capi.lib().nwg_abi_version() == 4


def test_workload_generator_is_seeded_and_distinct():
    pkg = importlib.import_module("neuroevolutionary-wordle_b200")
    w = pkg.workload
    a = w.synthetic_words(512, 0)
    b = w.synthetic_words(512, 0)
    assert (a == b).all()
    assert len({r.tobytes() for r in a}) == 512
    assert a.max() < 26
    sub = w.secret_subset(512, 256, 0)
    off, words = w.fixed_cell_lists(64, 64, sub, 0)
    assert off[-1] == len(words) == 64 * 64
    for c in range(64):
        cell = words[off[c]:off[c + 1]]
        assert len(set(cell.tolist())) == 64
        assert set(cell.tolist()) <= set(sub.tolist())
    off2, words2 = w.loguniform_cell_lists(100, 32, 1024, w.secret_subset(4739, 2315, 0), 0)
    sizes = (off2[1:] - off2[:-1]).astype(int)
    assert sizes.min() >= 32 and sizes.max() <= 1024


@pytest.mark.parametrize("a,expected", [(512, 339968), (4739, 661220), (1, 301132)])
def test_stride(a, expected):
    pkg = importlib.import_module("neuroevolutionary-wordle_b200")
    assert pkg.capi.genome_stride_bytes(a) == expected
