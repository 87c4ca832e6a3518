"""Failure detection without a GPU fault.

- A device allocation made to fail on the host (uc_ctx_set_faults
  fail_alloc_after): the call returns UC_ENOMEM and the same context then
  compacts the job bit-exactly.
- The HEC contraction's bounded rounds run out on the device (a round cap of
  1 on lists that need more): the device sets its timeout flag, the call
  returns UC_ETIMEOUT under hec_strict (and finishes by pointer jumping
  without it), and the same context then compacts the job bit-exactly.

The reference has no error path besides exit(1) on a file it cannot open
(driver.cpp:262-265), and spins without bound in its matching
(heuristics.h:119-147)."""
import pytest
import torch

from tests.cases import distinct_path, shuffled, text_of, walk_kmers
from unitigcoarsening_b200 import Compactor, api, synth

pytestmark = pytest.mark.gpu

UC_ENOMEM, UC_ETIMEOUT = 2, 4


def _lines(b: bytes):
    return sorted(b.split(b"\n")[:-1])


@pytest.fixture(scope="module")
def job(oracle):
    text = synth.make_text(synth.small_plain(seed=3, length=300_000), 31).numpy().tobytes()
    want, n, _ = oracle.compact(text, 31)
    return text, _lines(want), n


def _dev(text: bytes):
    return torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()


@pytest.mark.parametrize("nth", [1, 2, 3])
def test_failed_allocation_is_enomem_and_context_recovers(job, nth):
    text, want, _ = job
    d = _dev(text)
    with Compactor(0) as c:  # a fresh context: its buffers are allocated on demand
        c.set_faults(fail_alloc_after=nth)
        with pytest.raises(api.UCError) as ei:
            c.compact(d, 31, 8)
        assert ei.value.status == UC_ENOMEM, str(ei.value)
        c.set_faults()
        out = c.compact(d, 31, 8)
        torch.cuda.synchronize()
        assert _lines(out.cpu().numpy().tobytes()) == want


def test_failed_allocation_on_host_path(job):
    text, want, _ = job
    with Compactor(0) as c:
        # resident only: by default a host job that cannot allocate runs
        # streamed instead (tests/test_gpu_streamed.py)
        c.set_streaming(api.STREAM_NEVER)
        c.set_faults(fail_alloc_after=1)  # the device text buffer of the host path
        with pytest.raises(api.UCError) as ei:
            c.compact_host(text, 31, 8)
        assert ei.value.status == UC_ENOMEM, str(ei.value)
        c.set_faults()
        out = c.compact_host(text, 31, 8)
        assert _lines(out.numpy().tobytes()) == want


def test_hec_rounds_run_out_fused_path(job):
    text, want, _ = job
    d = _dev(text)
    with Compactor(0) as c:
        c.set_tuning(contract_method=api.CONTRACT_HEC)
        # strict: the device-side round budget runs out -> UC_ETIMEOUT
        c.set_faults(hec_round_cap=1, hec_strict=True)
        with pytest.raises(api.UCError) as ei:
            c.compact(d, 31, 8)
        assert ei.value.status == UC_ETIMEOUT, str(ei.value)
        # not strict: the same cap finishes the lists by pointer jumping
        c.set_faults(hec_round_cap=1)
        out = c.compact(d, 31, 8)
        torch.cuda.synchronize()
        assert _lines(out.cpu().numpy().tobytes()) == want
        # no faults: HEC alone, on the same context
        c.set_faults()
        out = c.compact(d, 31, 8)
        torch.cuda.synchronize()
        assert _lines(out.cpu().numpy().tobytes()) == want


def test_hec_rounds_run_out_phase_api(comp, oracle):
    k = 31
    seq = distinct_path(600, k, seed=5)
    text = text_of(shuffled(walk_kmers(seq, k), 3))
    d = _dev(text)
    keys = comp.load_kmers(d, k)
    succ, pred = comp.assemble_pruned_graph(keys, k, 8)
    try:
        comp.set_faults(hec_round_cap=1, hec_strict=True)
        with pytest.raises(api.UCError) as ei:
            comp.coarsen_de_bruijn_full_cycle(keys, succ, pred, k, method=api.CONTRACT_HEC)
        assert ei.value.status == UC_ETIMEOUT, str(ei.value)
    finally:
        comp.set_faults()
    head, rank, cyc = comp.coarsen_de_bruijn_full_cycle(keys, succ, pred, k, method=api.CONTRACT_HEC)
    out = comp.write_unitigs(keys, succ, head, rank, k)
    torch.cuda.synchronize()
    assert _lines(out.cpu().numpy().tobytes()) == [seq.encode()]
    assert cyc == 0
