"""The C++ compat layer (include/nwg_slab_device_shim.hpp): the reference's slab_device API on the C ABI.

Host (no GPU): compiled against the reference's own headers, the shim defines every function
genetic_algorithm/device/slab_runtime.hpp:119-186 declares. B200: tests/shim_driver.cu, a caller written only
against the reference's API and linked with libnwg.so through the shim, walks the reference CLI's calls
(cli/run_genetic_algorithm.cu: create, bootstrap, evaluate, advance with both callbacks and an injection asked
for by the shard-release callback, checkpoint + asynchronous write + resume, restore + resume); its fitness
equals the reference runtime's bit for bit, and its children equal the reference runtime's and this library's
direct API's, byte for byte.
"""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import build as oracle_build
from oracle import pyoracle as O

ROOT = Path(__file__).resolve().parent.parent
DRIVER = ROOT / "oracle" / "_ref" / "shim_driver"


def _declared_reference_functions() -> list[str]:
    text = (oracle_build.REFERENCE_ROOT / "src/genetic_algorithm/device/slab_runtime.hpp").read_text()
    names = set(re.findall(r"^(?:bool|void|const char \*)\s+(\w+)\(", text, flags=re.M))
    names |= {"RuntimeCheckpointAsyncWriter::" + m for m in ("TryStartWrite", "IsWriteInProgress",
                                                              "TryCollectFinishedWrite", "TryWaitForWrite")}
    return sorted(names)


@pytest.mark.skipif(not oracle_build.reference_present(), reason="reference headers not present")
def test_shim_defines_every_reference_entry_point(tmp_path):
    src = tmp_path / "shim_impl.cu"
    src.write_text('#define NWG_SLAB_DEVICE_SHIM_IMPLEMENTATION\n#include "nwg_slab_device_shim.hpp"\n')
    obj = tmp_path / "shim_impl.o"
    subprocess.run([oracle_build.NVCC, *oracle_build.ARCH, "-std=c++20", "-c", "-I",
                    str(oracle_build.REFERENCE_ROOT / "src"), "-I", str(ROOT / "include"), str(src), "-o", str(obj)],
                   check=True)
    defined = subprocess.run(["nm", "-C", "--defined-only", str(obj)], check=True, capture_output=True,
                             text=True).stdout
    names = _declared_reference_functions()
    assert len(names) >= 20
    missing = [n for n in names if f"slab_device::{n}(" not in defined]
    assert not missing, missing


def _fnv(data: np.ndarray) -> str:
    h = 1469598103934665603
    for b in data.tobytes():
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


def _parse(out: str) -> dict:
    lines = {}
    for line in out.strip().splitlines():
        key, *rest = line.split()
        lines[key] = rest
    return lines


@pytest.mark.gpu
@pytest.mark.skipif(not DRIVER.exists() or O.ref_ckpt() is None, reason="shim driver or reference library not built")
@pytest.mark.parametrize("actions,injected,slots,population,columns,boot_seed,boot_index,seed", [
    (20, 3, 18, 9, 3, 173, 4, 29), (200, 0, 32, 16, 4, 5, 0, 99)])
def test_reference_api_through_the_shim(tmp_path, actions, injected, slots, population, columns, boot_seed,
                                        boot_index, seed):
    import importlib

    from tests import helpers as H

    nwg = importlib.import_module("neuroevolutionary-wordle_b200")
    capi = nwg.capi
    rng = np.random.default_rng(actions + injected)
    while True:
        catalog = H.synthetic_words(rng, actions + injected)
        if all(O.hint_grid_group(w) is not None for w in catalog):
            break
    cat_file = tmp_path / "catalog.bin"
    cat_file.write_bytes(np.ascontiguousarray(catalog, np.uint8).tobytes())
    run = subprocess.run([str(DRIVER), str(cat_file), str(actions), str(injected), str(slots), str(population),
                          str(columns), str(boot_seed), str(boot_index), str(seed), str(tmp_path / "ck.bin")],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    got = _parse(run.stdout)
    assert "ok" in got
    stride = capi.genome_stride_bytes(actions)
    assert got["layout"] == [str(actions), str(stride), str(slots), str(population), str(columns)]

    # evaluation: the reference runtime on the same inputs
    counts = capi.word_counts(training=actions, action_space=actions)
    rc = capi.RuntimeConfig()
    rc.genotype_slab_byte_budget_bytes = slots * stride
    rc.generation_byte_budget_bytes = population * stride
    rc.action_count, rc.population_size_ceiling, rc.grid_column_count = actions, population, columns
    fit = np.zeros(population, np.float32)
    evals = np.zeros(population, np.uint32)
    has = np.zeros(population, np.uint8)
    summary = capi.FitnessSummary()
    assert O.ref_ckpt().refckpt_runtime_evaluate(C.addressof(rc), catalog.ctypes.data, len(catalog), population,
                                                 boot_seed, boot_index, C.addressof(counts), None, fit.ctypes.data,
                                                 evals.ctypes.data, has.ctypes.data, C.addressof(summary)) == 1
    assert got["fitness"] == [f"{v:08x}" for v in fit.view(np.uint32)]
    assert int(got["summary"][2]) == summary.best_index and int(got["summary"][3]) == summary.generation_index

    # the advance, by the reference runtime: prepare with the same injection, then resume
    cfg = capi.assembly_config(radius=1, p=0.01, sigma=0.02)
    pending = capi.PendingInjection(injected > 0, actions if injected else 0, injected)
    ref_ck = tmp_path / "ref.bin"
    assert O.ref_ckpt().refckpt_runtime_capture(C.addressof(rc), catalog.ctypes.data, len(catalog), population,
                                                boot_seed, boot_index, seed, C.addressof(counts), C.addressof(cfg),
                                                C.addressof(pending), None, 0, str(ref_ck).encode()) == 1
    cap = 64 * capi.genome_stride_bytes(actions + injected)
    buf = np.zeros(cap, np.uint8)
    n, st = C.c_size_t(), C.c_size_t()
    assert O.ref_ckpt().refckpt_runtime_resume(str(ref_ck).encode(), catalog.ctypes.data, len(catalog),
                                               buf.ctypes.data, cap, C.byref(n), C.byref(st)) == 1
    ref_children = buf[:n.value * st.value].reshape(n.value, st.value)
    advanced = got["advanced"]
    assert int(advanced[0]) == boot_index + 1 and int(advanced[1]) == n.value
    assert advanced[2:] == [_fnv(c) for c in ref_children]
    assert got["callbacks"][:2] == ["1", "1"] and int(got["callbacks"][2]) == n.value
    assert int(got["grown"][0]) == actions + injected

    # the checkpointed step: resumed in place, restored from the file, and this library's direct API agree
    assert got["resumed"] == got["restored"]
    G = importlib.import_module("tests.gpu_util")
    G.upload_catalog_everywhere(catalog)
    rt = nwg.Runtime(actions, population, columns, slab_generations=slots / population)
    rt.bootstrap(population, seed=boot_seed, generation_index=boot_index)

    def release(_rt, _counts, pend, _user):
        if injected:
            pend[0].enabled = True
            pend[0].first_catalog_word_index = actions
            pend[0].injection_count = injected
        return True

    rt.advance(seed, counts, config=cfg, shard_release=release)
    grown = capi.word_counts(training=actions, action_space=actions + injected)
    rt.checkpoint(seed + 1, grown, config=cfg)
    rt.assemble()
    gen = rt.current_generation()
    direct = [_fnv(rt.download_slot(int(s))) for s in gen["slots"]]
    assert got["resumed"][2:] == direct
    assert got["status"][0] == "0"
    rt.close()
