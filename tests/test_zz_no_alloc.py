"""The allocation-free hamiltonian entry against the regular one.

Callers that cannot let the library call cudaMalloc (a host code that owns the whole device
memory pool, a caller inside another framework's memory pool, a loop where an allocation's
implicit synchronisation would stall) use rsdft_gpu_hamiltonian_noalloc_d, whose only scratch
is a fixed array compiled into the library.  The first call comes on a fresh context, before
anything else has touched its workspaces, and must leave them unallocated; two calls in a row,
with different inputs and band counts, must give the regular entry's result within the FP64
tolerance (1e-12 of max|H psi|); oversized requests and bad leading dimensions must be refused
before any work.  This file is collected last so a failure here leaves every other test
already run.
"""
import ctypes as C

import numpy as np
import pytest

from rsdft_develop_b200 import api, synth

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_noalloc_hamiltonian_first_call_allocates_nothing_and_matches_regular_entry_twice():
    torch = pytest.importorskip("torch")
    prob = synth.make_problem("c0")
    with api.BandUpdate(prob) as g:
        xs = [torch.from_numpy(synth.random_wavefunctions(seed, nb, prob.ng)).cuda() for seed, nb in ((91, 7), (92, 5))]
        outs = [torch.full_like(x, float("nan")) for x in xs]
        torch.cuda.synchronize()
        before = g.profile_get("workspace_bytes")[2]
        for x, out in zip(xs, outs):  # the allocation-free entry first, on a fresh context
            g.hamiltonian_noalloc_device(x.data_ptr(), out.data_ptr(), x.shape[0])
            g.synchronize()
        assert g.profile_get("workspace_bytes")[2] == before
        for call, (x, out) in enumerate(zip(xs, outs)):
            ref = torch.zeros_like(x)
            g.hamiltonian_device(x.data_ptr(), ref.data_ptr(), x.shape[0])
            g.synchronize()
            r = ref.cpu().numpy()
            o = out.cpu().numpy()
            assert np.all(np.isfinite(o)), call
            assert np.max(np.abs(o - r)) <= TOL * np.max(np.abs(r)), call


def test_noalloc_hamiltonian_rejects_oversized_request_and_bad_ld():
    prob = synth.make_problem("c0")
    with api.BandUpdate(prob) as g:
        slots = prob.nzlma  # s+p atoms: 4 projectors each, no padding
        nb = 524288 // slots + 1
        with pytest.raises(api.RsdftError) as e:
            # rejected on the host before any device access
            api._call(g.lib.rsdft_gpu_hamiltonian_noalloc_d, 1, 1, C.c_void_p(256), C.c_void_p(256), prob.ng, nb)
        assert e.value.code == -1
        assert "exceed the fixed scratch" in str(e.value)
        with pytest.raises(api.RsdftError) as e:
            api._call(g.lib.rsdft_gpu_hamiltonian_noalloc_d, 1, 1, C.c_void_p(256), C.c_void_p(256), -prob.ng, 1)
        assert e.value.code == -1
