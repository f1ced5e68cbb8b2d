"""Differentiable, batched and complex64 expectation on the GPU.

Gradients are checked against the FP64 oracle (per-term <P_k>, H psi) and
against central finite differences (h = 1e-6); batched results against the
per-call plan path and the oracle; complex64 storage against the FP64 oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import random_operator

pytestmark = pytest.mark.gpu


def hermitian_op(rng, n, T, p=0.3):
    n, x, z, c = random_operator(rng, n, T, p)
    return n, x, z, rng.normal(size=T).astype(np.complex128)


def test_autograd_matches_oracle_and_finite_differences(cuda, oracle):
    torch = cuda
    from wolfgang_b200.expectation import ExpectationPlan, expectation

    rng = np.random.default_rng(41)
    n, x, z, c = hermitian_op(rng, 10, 300)
    psi_np = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi_np /= np.linalg.norm(psi_np)
    plan = ExpectationPlan((n, x, z, c))
    coeffs = torch.tensor(c.real, dtype=torch.float64, device="cuda", requires_grad=True)
    psi = torch.tensor(psi_np, dtype=torch.complex128, device="cuda", requires_grad=True)
    E = expectation(plan, coeffs, psi)
    E.backward()
    assert abs(E.item() - oracle.expectation(n, x, z, c, psi_np).real) <= 1e-12
    assert torch.max(torch.abs(coeffs.grad.cpu() - torch.from_numpy(oracle.term_expectations(n, x, z, psi_np)))) <= 1e-12
    hp = oracle.hpsi(n, x, z, c, psi_np)
    assert np.max(np.abs(psi.grad.cpu().numpy() - 2 * hp)) <= 1e-12

    h = 1e-6
    with torch.no_grad():
        for k in (0, 7, 123):
            e = torch.zeros_like(coeffs)
            e[k] = h
            fd = (expectation(plan, coeffs + e, psi) - expectation(plan, coeffs - e, psi)) / (2 * h)
            assert abs(fd.item() - coeffs.grad[k].item()) <= 1e-7
        for trial in range(3):
            v = torch.randn(1 << n, dtype=torch.complex128, device="cuda")
            fd = (expectation(plan, coeffs, psi + h * v) - expectation(plan, coeffs, psi - h * v)) / (2 * h)
            analytic = torch.real(torch.vdot(psi.grad, v))
            assert abs(fd.item() - analytic.item()) <= 1e-6 * max(1.0, abs(analytic.item()))
    plan.close()


def test_complex64_storage_fp64_accumulation(cuda, oracle):
    torch = cuda
    from wolfgang_b200.expectation import ExpectationPlan

    rng = np.random.default_rng(64)
    n, x, z, c = hermitian_op(rng, 16, 2000)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    p64 = psi.astype(np.complex64)
    plan = ExpectationPlan((n, x, z, c))
    res, ev, hp = plan.run(torch.from_numpy(p64).cuda(), terms=True, hpsi=True)
    # same input (the complex64 values widened), FP64 accumulation: 1e-12 vs the oracle on those values
    assert abs(complex(res[0].item(), res[1].item()) - oracle.expectation(n, x, z, c, p64)) <= 1e-12
    assert np.max(np.abs(ev.cpu().numpy() - oracle.term_expectations(n, x, z, p64))) <= 1e-12
    # against the complex128 state: the storage rounding only (relative 1e-6)
    e128 = oracle.expectation(n, x, z, c, psi)
    assert abs(res[0].item() - e128.real) <= 1e-6 * max(1.0, abs(e128))
    plan.close()


def test_batched_uneven_pairs_match_per_call_and_oracle(cuda, oracle):
    torch = cuda
    from wolfgang_b200.expectation import ExpectationBatch, ExpectationPlan

    rng = np.random.default_rng(512)
    ops, psis, plans = [], [], []
    for i in range(24):
        n = int(rng.integers(3, 15))
        T = int(np.exp(rng.uniform(np.log(5), np.log(600))))
        op = hermitian_op(rng, n, T, 0.3)
        psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        psi /= np.linalg.norm(psi)
        ops.append(op)
        psis.append(torch.from_numpy(psi).cuda())
        plans.append(ExpectationPlan(op))
    batch = ExpectationBatch(plans, psis, gradients=True)
    batch.run()
    torch.cuda.synchronize()
    first = batch.values.clone()
    batch.replay()  # captured CUDA graph
    torch.cuda.synchronize()
    assert torch.equal(first, batch.values)
    for i, (op, plan, psi) in enumerate(zip(ops, plans, psis)):
        res, ev, hp = plan.run(psi, terms=True, hpsi=True)
        torch.cuda.synchronize()
        assert torch.equal(res, batch.values[i])
        assert torch.equal(ev, batch.term_values[i][: plan.T])
        assert torch.equal(hp, batch.hpsi[i])
        if i < 6:
            n, x, z, c = op
            pn = psi.cpu().numpy()
            assert abs(complex(res[0].item(), res[1].item()) - oracle.expectation(n, x, z, c, pn)) <= 1e-12
            assert np.max(np.abs(hp.cpu().numpy() - oracle.hpsi(n, x, z, c, pn))) <= 1e-12
    batch.close()
    for p in plans:
        p.close()


def test_plan_rejects_masks_beyond_num_qubits(cuda):
    torch = cuda
    from wolfgang_b200.expectation import ExpectationPlan

    x = np.array([[1 << 5]], np.uint64)
    z = np.zeros((1, 1), np.uint64)
    with pytest.raises(ValueError, match="num_qubits"):
        ExpectationPlan((4, x, z, np.ones(1, np.complex128)))
