"""Bounded device waits, driven on the GPU without a fault.

Every wait between the roles of the tensor-memory kernel (row loads, tensor
memory slots, accumulators) gives up after the context's wait limit, sets an
error bit, and the kernel drains its own copies and MMAs, frees its tensor
memory and returns; the call reports KG_ERR_TIMEOUT.  The reference has no
device waits: its failures end the process with `[ERROR] ...` and exit code 1
(die(), src/kgwas_utils.hpp:34-37), which the kgwas program maps
KG_ERR_TIMEOUT to.

Here the row producer of every CTA stops after its first row load (the test
hook kg_inject_stall), so the unpack warps' waits for the next rows can never
be satisfied and run out after a 1 ms limit.  The same context then runs a
normal call, with the short limit still in force and again with the default,
and must match the FP64 oracle.
"""
import time

import numpy as np
import pytest

from oracle import oracle as O
from supergwas_b200 import api, synth
from test_gpu_parity import check_against_oracle

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_context_stays_usable(built):
    import torch
    ds = synth.simulate(n=1000, m=100_000, S=8, r=16, n_causal=20, missing=0.05, seed=61)
    X = ds.packed_overlap()
    m, wpk = X.shape
    o = O.cols_stats(X, ds.n, ds.U, ds.y, 0.0)
    dx = torch.from_numpy(X.view(np.int64)).cuda()
    st = torch.cuda.Stream()
    with api.Kgwas(precision="split", corr_threshold=0.0, log10_thresh=2.0) as g:
        g.set_structure(ds.U, ds.y)
        g.set_wait_limit(1_000_000)  # 1 ms
        g.inject_stall(1)            # each CTA loads one box of rows, then stops
        t0 = time.perf_counter()
        g.launch_device(dx.data_ptr(), m, wpk, st.cuda_stream)
        with pytest.raises(api.KgError) as ei:
            g.fetch()
        dt = time.perf_counter() - t0
        assert ei.value.code == 5, str(ei.value)  # KG_ERR_TIMEOUT
        assert g.last_kernel() == "ts"
        assert dt < 1.5, dt  # the 1 ms limit was in force, not the 2 s default
        torch.cuda.synchronize()  # the context and the device are fine

        # a normal call on the same context, the short limit still set
        res = g.run_host(X, stats=True)
        assert g.last_kernel() == "ts"
        check_against_oracle(res, o, "split", 0.0, 2.0)

        # and with the default limit again
        g.set_wait_limit(0)
        g.launch_device(dx.data_ptr(), m, wpk, st.cuda_stream)
        r2 = g.fetch()
        assert r2.n_tested == o["n_tested"]
        assert np.array_equal(r2.hits, res.hits)
