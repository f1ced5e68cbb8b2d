"""Parity at the benchmark configurations' full sizes.

* config 2 -- 32,768 x 16,384 products on 100 qubits, matmul + simplify: the
  whole device result (every one of its ~5e8 survivors) is compared with the
  oracle, bit for bit, one key range at a time: the ranges are cut at every
  2^23-th survivor of the device result, plus the empty ranges before the
  first and after the last key, and each range's oracle result (survivor count
  and a digest of keys and coefficient bits) must equal the device slice.
* config 3 -- the 262,144-term commutation matrix (row blocks against the
  oracle, symmetry and the diagonal across the matrix) and group_commuting at
  262,144 terms (qwc) and 32,768 terms (full), against the reference core.
* config 4 -- 26 qubits, 20,000 terms: sampled <P_k> and H psi against the
  oracle (<= 1e-12), E against two identities of oracle-checked values, and
  central finite differences (h = 1e-6) along random state directions and
  coefficients.  (The oracle's E over all terms would be 20,000 x 2^25 pair
  steps; the identities E = sum_k c_k <P_k> and E = <psi|H psi> bind it to
  the checked values instead.)
* config 5 -- all 512 uneven pairs, complex128 and complex64 states: every
  pair's term values on a sample of its terms (all of them where the oracle's
  cost allows), sampled H psi and, where affordable, E against the oracle.

The oracle runs in spawned worker processes (tests/fullsize_oracle.py).
"""

from __future__ import annotations

import ctypes
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from tests import fullsize_oracle as FO
from tests import gpu_util as G
from wolfgang_b200 import capi

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

W = workloads = FO.workloads()


def _download(ptr, offset_bytes, nbytes, dtype):
    out = np.empty(nbytes // np.dtype(dtype).itemsize, dtype)
    if nbytes:
        capi.call("wg_memcpy_dtoh", 0, out.ctypes.data, ptr + offset_bytes, nbytes, None)
    return out


# ----------------------------------------------------------------- config 2

def test_config2_full_products_bit_exact(cuda):
    A, B = workloads.klocal_pair_100q()
    n, w = 100, 2
    nl, nr = len(A[3]), len(B[3])
    with FO.pool() as pool:  # spawned before the device work below
        pool.map(FO.digest, [np.zeros(1)])  # start the workers
        ax, az, ac = G.operator_on_device(A[1], A[2], A[3])
        bx, bz, bc = G.operator_on_device(B[1], B[2], B[3])
        ox, oz, oc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        U = ctypes.c_size_t()
        capi.call("wg_pauli_products", 0, w, ax.data_ptr(), az.data_ptr(), ac.data_ptr(), nl, bx.data_ptr(),
                  bz.data_ptr(), bc.data_ptr(), nr, capi.WG_PRODUCTS_SIMPLIFY, 1e-12, 0.0, ctypes.byref(ox),
                  ctypes.byref(oz), ctypes.byref(oc), ctypes.byref(U), None)
        U = U.value
        try:
            assert U == 500_565_508  # every range below is also checked against the oracle
            R = 1 << 23
            cuts = list(range(0, U, R)) + [U]

            def key(p):
                xs = _download(ox.value, p * 16, 16, np.uint64)
                zs = _download(oz.value, p * 16, 16, np.uint64)
                return np.array([xs[0], zs[0], xs[1], zs[1]], np.uint64)

            lo_all = np.zeros(4, np.uint64)
            hi_all = np.full(4, np.iinfo(np.uint64).max, np.uint64)
            bounds = [key(p) for p in cuts[:-1]]
            last = key(U - 1)
            assert not np.array_equal(last, hi_all)
            after_last = last.copy()  # the successor of the last key in canonical order
            for i in range(3, -1, -1):
                if after_last[i] != np.iinfo(np.uint64).max:
                    after_last[i] += np.uint64(1)
                    break
                after_last[i] = 0
            ranges = [(lo_all, bounds[0], 16)]
            ranges += [(bounds[k], bounds[k + 1] if k + 1 < len(bounds) else after_last, cuts[k + 1] - cuts[k] + 16)
                       for k in range(len(bounds))]
            ranges += [(after_last, hi_all, 16)]
            pending = pool.map_async(FO.products_range, ranges, chunksize=1)

            def device_slice(k):
                p0, p1 = cuts[k], cuts[k + 1]
                xs = _download(ox.value, p0 * 16, (p1 - p0) * 16, np.uint64).reshape(-1, 2)
                zs = _download(oz.value, p0 * 16, (p1 - p0) * 16, np.uint64).reshape(-1, 2)
                cs = _download(oc.value, p0 * 16, (p1 - p0) * 16, np.float64).view(np.complex128)
                return p1 - p0, FO.digest(xs, zs, cs)

            with ThreadPoolExecutor(8) as ex:
                mine = [(0, FO.digest(np.zeros((0, 2), np.uint64), np.zeros((0, 2), np.uint64),
                                      np.zeros(0, np.complex128)))]
                mine += list(ex.map(device_slice, range(len(cuts) - 1)))
                mine += [mine[0]]
            theirs = pending.get(timeout=1800)
        finally:
            for p in (ox, oz, oc):
                if p.value:
                    capi.call("wg_free", 0, p.value, None)
    assert len(theirs) == len(mine) == len(cuts) + 1
    bad = [k for k, (a, b) in enumerate(zip(mine, theirs)) if a != b]
    assert not bad, f"key ranges differing from the oracle: {bad[:10]} (device, oracle): " \
                    f"{[(mine[k][0], theirs[k][0]) for k in bad[:5]]}"
    assert sum(t[0] for t in theirs) == U


# ----------------------------------------------------------------- config 3

def test_config3_commutation_matrix_full_size(cuda, oracle):
    torch = cuda
    n, x, z, _ = workloads.sparse_operator_128q()
    T = len(x)
    pitch = (T + 31) // 32
    dx, dz = G.dev(x), G.dev(z)
    bits = torch.empty(T * pitch, dtype=torch.int32, device="cuda")
    capi.call("wg_commutation_bits", 0, 2, dx.data_ptr(), dz.data_ptr(), T, dx.data_ptr(), dz.data_ptr(), T,
              bits.data_ptr(), pitch, 0, None)
    torch.cuda.synchronize()
    mat = bits.view(T, pitch)
    rng = np.random.default_rng(3)
    # row blocks (first, last, random) against the oracle
    for r0 in (0, T - 256, int(rng.integers(0, T - 256))):
        got = G.unpack_bits(mat[r0:r0 + 256].cpu().numpy().view(np.uint32), T)
        assert np.array_equal(got, oracle.commutes(n, (x[r0:r0 + 256], z[r0:r0 + 256]), (x, z)))
    # symmetry of 2,048 x 2,048 blocks anywhere in the matrix, and the diagonal
    for _ in range(4):
        r0, c0 = (int(v) * 32 for v in rng.integers(0, (T - 2048) // 32, size=2))
        rows = G.unpack_bits(mat[r0:r0 + 2048, c0 // 32:(c0 + 2048) // 32].cpu().numpy().view(np.uint32), 2048)
        cols = G.unpack_bits(mat[c0:c0 + 2048, r0 // 32:(r0 + 2048) // 32].cpu().numpy().view(np.uint32), 2048)
        assert np.array_equal(rows, cols.T)
    diag = torch.arange(T, device="cuda")
    words = mat[diag, diag // 32]
    assert bool(torch.all(((words >> (diag % 32).to(torch.int32)) & 1) == 1))
    # the total from the popcount consumer equals the row counts' sum
    total = ctypes.c_uint64()
    rc = torch.zeros(T, dtype=torch.int64, device="cuda")
    capi.call("wg_bits_count", 0, bits.data_ptr(), T, T, pitch, rc.data_ptr(), None, ctypes.byref(total), None)
    assert int(rc.sum().item()) == total.value
    del bits


def _device_groups(n, x, z, mode):
    T = len(x)
    dx, dz = G.dev(x), G.dev(z)
    order = np.zeros(T, np.uintp)
    sizes = np.zeros(T, np.uintp)
    ng = ctypes.c_size_t()
    capi.call("wg_group_commuting", 0, (n + 63) // 64, T, dx.data_ptr(), dz.data_ptr(), 1 if mode == "full" else 0,
              order.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)),
              sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)), ctypes.byref(ng), None)
    return order, sizes[: ng.value]


@pytest.mark.parametrize("mode,T", [("qwc", 262144), ("full", 32768)])
def test_config3_grouping_matches_reference_core(cuda, reference, mode, T):
    n, x, z, c = workloads.sparse_operator_128q()
    x, z, c = x[:T], z[:T], c[:T]
    order, sizes = _device_groups(n, x, z, mode)
    want = reference.group_commuting(n, x, z, c, mode)
    assert [int(s) for s in sizes] == [len(g[2]) for g in want]
    order = order.astype(np.int64)
    assert np.array_equal(x[order], np.concatenate([g[0] for g in want]))
    assert np.array_equal(z[order], np.concatenate([g[1] for g in want]))
    assert np.ascontiguousarray(c[order]).tobytes() == np.concatenate([g[2] for g in want]).tobytes()


# ----------------------------------------------------------------- config 4

def test_config4_26_qubits_values_gradients_and_finite_differences(cuda, oracle):
    torch = cuda
    from wolfgang_b200.expectation import ExpectationPlan

    n, x, z, c = workloads.xpattern_operator(n=26)
    psi_np = workloads.state_26q()
    T = len(c)
    plan = ExpectationPlan((n, x, z, c))
    psi = torch.from_numpy(psi_np).cuda()
    res, ev, hp = plan.run(psi, terms=True, hpsi=True)
    torch.cuda.synchronize()
    E = complex(res[0].item(), res[1].item())
    ev = ev.cpu().numpy()
    rng = np.random.default_rng(26)
    sample = rng.choice(T, size=64, replace=False)
    want = oracle.term_expectations(n, x[sample], z[sample], psi_np)
    assert np.max(np.abs(ev[sample] - want)) <= 1e-12
    idx = rng.integers(0, 1 << n, size=256, dtype=np.uint64)
    hp_s = hp[torch.from_numpy(idx.astype(np.int64)).cuda()].cpu().numpy()
    assert np.max(np.abs(hp_s - oracle.hpsi_at(n, x, z, c, psi_np, idx))) <= 1e-12
    # E is bound to the checked values: sum_k c_k <P_k> and <psi|H psi>
    assert abs(E.real - math.fsum(c.real * ev)) <= 1e-12
    assert abs(E.imag) <= 1e-12
    assert abs(E - complex(torch.vdot(psi, hp).item())) <= 1e-12

    h = 1e-6
    coeffs = torch.from_numpy(c.real.copy()).cuda()

    def energy(cf, ps):
        plan.set_coefficients(cf.to(torch.complex128))
        r, _, _ = plan.run(ps)
        return r[0].item()

    for k in rng.choice(T, size=8, replace=False):
        e = torch.zeros_like(coeffs)
        e[int(k)] = h
        fd = (energy(coeffs + e, psi) - energy(coeffs - e, psi)) / (2 * h)
        assert abs(fd - ev[int(k)]) <= 1e-7
    for _ in range(3):
        v = torch.randn(1 << n, dtype=torch.complex128, device="cuda")
        v /= torch.linalg.vector_norm(v)
        fd = (energy(coeffs, psi + h * v) - energy(coeffs, psi - h * v)) / (2 * h)
        analytic = 2.0 * torch.real(torch.vdot(v, hp)).item()  # dE along v = 2 Re<v|H psi>
        assert abs(fd - analytic) <= 1e-6 * max(1.0, abs(analytic))
    plan.close()


# ----------------------------------------------------------------- config 5

@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_config5_all_512_pairs_against_oracle(cuda, dtype):
    torch = cuda
    from wolfgang_b200.expectation import ExpectationBatch, ExpectationPlan

    pairs = workloads.uneven_pairs(512)
    npdt = np.complex128 if dtype == "c128" else np.complex64
    rng = np.random.default_rng(5)
    jobs = []
    budget = 1 << 25  # oracle pair steps per pair: T_sampled * 2^(n-1)
    for n, T, seed in pairs:
        m = T if T << (n - 1) <= budget else max(4, budget >> (n - 1))
        sample = np.sort(rng.choice(T, size=min(m, T), replace=False))
        idx = rng.integers(0, 1 << n, size=8, dtype=np.uint64)
        jobs.append((n, T, seed, sample, idx, dtype, m >= T))
    with FO.pool() as pool:
        pending = pool.map_async(FO.pair_term_values, jobs, chunksize=1)
        plans, psis, ops = [], [], []
        for n, T, seed in pairs:
            op = workloads.uneven_pair_operator(n, T, seed)
            ops.append(op)
            plans.append(ExpectationPlan(op))
            psis.append(torch.from_numpy(workloads.uneven_pair_state(n, seed, npdt)).cuda())
        batch = ExpectationBatch(plans, psis, gradients=True)
        batch.run()
        torch.cuda.synchronize()
        oracle_out = pending.get(timeout=3600)
    worst_term, worst_hp, worst_e, full_pairs = 0.0, 0.0, 0.0, 0
    for p, ((n, T, seed), op, job, (vals, hp, E_full)) in enumerate(zip(pairs, ops, jobs, oracle_out)):
        sample, idx = job[3], job[4]
        ev = batch.term_values[p][:T].cpu().numpy()
        worst_term = max(worst_term, float(np.max(np.abs(ev[sample] - vals))))
        E = complex(batch.values[p, 0].item(), batch.values[p, 1].item())
        c = op[3].real
        assert abs(E.real - math.fsum(c * ev)) <= 1e-10 * max(1.0, math.fsum(np.abs(c * ev)))
        if dtype == "c128":
            got_hp = batch.hpsi[p][torch.from_numpy(idx.astype(np.int64)).cuda()].cpu().numpy()
            worst_hp = max(worst_hp, float(np.max(np.abs(got_hp - hp))))
        if E_full is not None:
            full_pairs += 1
            worst_e = max(worst_e, abs(E - E_full) / max(1.0, abs(E_full)))
    # FP64 accumulation either way: 1e-12 against the oracle on the same stored amplitudes
    assert worst_term <= 1e-12, worst_term
    assert worst_hp <= 1e-12, worst_hp
    assert worst_e <= 1e-10, worst_e
    assert full_pairs > 100  # the smaller pairs are checked whole
    batch.close()
    for pl in plans:
        pl.close()
