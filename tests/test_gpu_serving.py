"""GPU tests of the continuous-batching request loop (serving, the mixed-size request benchmark).

The contract under test: requests of mixed grid sizes arrive while others run,
join the next batch of their class, and each result equals the same request
computed alone (members are independent, so the comparison is exact), and the
FP64-plain results match the oracle flux.
"""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CLASSES = [(32, 9, 3, 4, skb_cuda.FLUX_FP64_PLAIN), (64, 17, 4, 4, skb_cuda.FLUX_FP64_PLAIN),
           (64, 17, 4, 4, skb_cuda.FLUX_SPLIT_TF32X3)]


def inputs_for(cls, seed):
    n, nz, targets = CLASSES[cls][:3]
    modes = orc.retained_modes(n, n)
    return orc.flux_inputs(modes, 3 + 3 * targets, 2 * (nz - 1) // 3, seed)


def alone(cls, x):
    n, nz, targets, _, mode = CLASSES[cls]
    return skb_cuda.Flux(n, nz, targets=targets, members=1, mode=mode).execute(x)


def test_partial_batch_equals_full_batch():
    n, nz, members = 32, 9, 4
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    xs = [orc.flux_inputs(modes, 15, nj, 40 + m) for m in range(members)]
    for mode in (skb_cuda.FLUX_FP64_PLAIN, skb_cuda.FLUX_SPLIT_TF32X3):
        flux = skb_cuda.Flux(n, nz, members=members, mode=mode)
        dt = flux.device_dtype
        din = skb_cuda.DeviceArray.from_numpy(np.concatenate(xs).astype(dt))
        dout = skb_cuda.DeviceArray(flux.output_elements * np.dtype(dt).itemsize)
        flux.execute_device(din.ptr, dout.ptr)
        skb_cuda.synchronize()
        full = dout.download(dt, flux.output_elements).reshape(members, -1)
        flux.execute_device(din.ptr, dout.ptr, members=2)
        skb_cuda.synchronize()
        part = dout.download(dt, flux.output_elements).reshape(members, -1)
        assert np.array_equal(part[:2], full[:2])


def test_mixed_stream_matches_alone_and_oracle():
    """Requests arrive while earlier batches run; how they group depends on
    timing, and no grouping may change a result."""
    server = skb_cuda.Server(CLASSES, hbm_budget_bytes=8 << 30, max_slots_per_class=2)
    rng = np.random.default_rng(7)
    classes = [int(rng.choice(len(CLASSES), p=[0.4, 0.4, 0.2])) for _ in range(24)]
    xs = [inputs_for(cls, 1000 + i) for i, cls in enumerate(classes)]
    jobs = [(cls, x, server.submit(cls, x)) for cls, x in zip(classes, xs)]
    results = [(cls, x) + server.wait(t, timeout=120) for cls, x, t in jobs]
    stats = server.stats()
    assert stats["completed"] == 24 and stats["submitted"] == 24
    assert 1 <= stats["batches"] <= 24
    for cls, x, out, latency in results:
        assert latency > 0
        assert np.array_equal(out, alone(cls, x))
        if CLASSES[cls][4] == skb_cuda.FLUX_FP64_PLAIN:
            n, nz, targets = CLASSES[cls][:3]
            assert orc.rel_l2_error(out, orc.flux(n, nz, x, targets=targets)) <= 1e-12
    server.close()


def test_burst_is_batched():
    """A burst queued while the loop is held runs as full batches of its class."""
    server = skb_cuda.Server(CLASSES, hbm_budget_bytes=8 << 30, max_slots_per_class=2)
    classes = [0] * 9 + [1] * 5 + [2] * 3
    xs = [inputs_for(cls, 2000 + i) for i, cls in enumerate(classes)]
    server.hold(True)
    tickets = [server.submit(cls, x) for cls, x in zip(classes, xs)]
    assert server.stats()["batches"] == 0
    server.hold(False)
    outs = [server.wait(t, timeout=120)[0] for t in tickets]
    # max_batch 4: 9 -> 4+4+1, 5 -> 4+1, 3 -> 3
    assert server.stats()["batches"] == 3 + 2 + 1
    for cls, x, out in zip(classes, xs, outs):
        assert np.array_equal(out, alone(cls, x))
    server.close()


def test_resident_states_and_admission():
    server = skb_cuda.Server(CLASSES[:1], hbm_budget_bytes=256 << 20, max_slots_per_class=1)
    x = inputs_for(0, 5)
    state = server.load_state(0, x)
    out = np.empty(server.sizes[0][1], np.complex128)
    got, _ = server.wait(server.submit_state(state, out))
    assert np.array_equal(got, alone(0, x))
    server.release_state(state)
    # Admission by HBM footprint: states are admitted while they fit the budget
    # left after the slots, and the next one is refused.
    st = server.stats()
    state_bytes = server.sizes[0][0] * 16
    fit = (st["budget_bytes"] - st["slot_bytes"]) // state_bytes
    assert fit > 0
    states = [server.load_state(0, x) for _ in range(fit)]
    with pytest.raises(MemoryError):
        server.load_state(0, x)
    server.release_state(states.pop())
    states.append(server.load_state(0, x))
    assert server.stats()["resident_states"] == fit
    server.close()
