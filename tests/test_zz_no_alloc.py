"""The allocation-free Hilbert sort (aarbf_hilbert_sort_noalloc) against the sort aarbf_build runs.

This entry point exists for callers that cannot allocate device memory while they run -- device
memory owned by the application's pool or arena, real-time loops that must not call the
allocator (it can synchronise the device). It keeps its working space in one fixed device array shared by every call. The test
calls it through the C ABI twice in a row on different inputs (so leftovers of the first call in
the shared array would show up in the second) and compares keys and permutation with
aarbf_build's, which must match exactly (integer outputs). It also checks that sizes beyond the
fixed maximum are refused.

The file is named to be collected last, so that a run stopping at the first failure has already
run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(n, seed):
    rng = np.random.default_rng(seed)
    p = np.clip(rng.normal(0.5, 0.2, (n, 3)), 0, 1)
    xyzw = np.concatenate([p, rng.uniform(0, 1, (n, 1))], 1).astype(np.float32)
    # exact duplicates and shared positions force the tie-break chain
    idx = rng.integers(0, n, n // 50)
    xyzw[idx[: len(idx) // 2]] = xyzw[0]
    xyzw[idx[len(idx) // 2:], :3] = xyzw[1, :3]
    return xyzw


def test_noalloc_sort_matches_build(aarbf_mod, orc):
    ctx = aarbf_mod.Context(0)
    try:
        for call, (n, seed) in enumerate([(200_000, 1), (aarbf_mod.NOALLOC_MAX_PARTICLES, 2)]):
            xyzw = _scene(n, seed)
            dom = orc.domain([xyzw])
            # the existing entry point
            ctx.set_particles(xyzw)
            ctx.set_domain(dom)
            ctx.build(0.01, 1)
            want_keys, want_perm = ctx.hilbert_keys()
            # the allocation-free one, on caller-owned device buffers
            d_in = ctx.device_alloc(16 * n)
            d_keys = ctx.device_alloc(8 * n)
            d_perm = ctx.device_alloc(4 * n)
            try:
                ctx.memcpy(d_in, xyzw, 16 * n)
                ctx.memset(d_keys, 0xff, 8 * n)
                ctx.memset(d_perm, 0xff, 4 * n)
                ctx.sync()
                aarbf_mod.hilbert_sort_noalloc(d_in, n, dom, d_keys, d_perm)
                keys = np.zeros(n, np.uint64)
                perm = np.zeros(n, np.uint32)
                ctx.memcpy(keys, d_keys, 8 * n)
                ctx.memcpy(perm, d_perm, 4 * n)
                ctx.sync()
            finally:
                for b in (d_in, d_keys, d_perm):
                    ctx.device_free(b)
            assert np.array_equal(keys, want_keys), f"call {call}: keys differ"
            assert np.array_equal(perm, want_perm), f"call {call}: permutation differs"
        # beyond the fixed maximum: refused before any GPU work
        with pytest.raises(aarbf_mod.AarbfError):
            aarbf_mod.hilbert_sort_noalloc(0, aarbf_mod.NOALLOC_MAX_PARTICLES + 1, np.zeros(8, np.float32), 0, 0)
        # host buffers instead of device memory: refused before any kernel is launched
        n = 1000
        xyzw = _scene(n, 3)
        keys = np.zeros(n, np.uint64)
        perm = np.zeros(n, np.uint32)
        with pytest.raises(aarbf_mod.AarbfError):
            aarbf_mod.hilbert_sort_noalloc(xyzw.ctypes.data, n, orc.domain([xyzw]), keys.ctypes.data,
                                           perm.ctypes.data)
        assert not keys.any() and not perm.any()
    finally:
        ctx.close()
