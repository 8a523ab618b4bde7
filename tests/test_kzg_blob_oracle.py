"""EIP-4844 blob oracle (orc_kzg_blob_commit / orc_kzg_blob_proof).  The
reference delegates to c-kzg-4844 with the mainnet setup, both absent, so
parity with its bytes is unpinned; these tests pin the algorithms instead:
the published evaluation-form formulas the device uses (barycentric y, the
quotient in evaluation form with its domain-point case) agree with the
oracle's coefficient-form route (Horner, synthetic division) on a small
domain, and the oracle's y agrees with a direct evaluation at full size."""
from __future__ import annotations

import random

import _blob as B
import _oracle as O

R = B.R


def spec_eval_form(evals_brp, z, n, w):
    """EIP-4844 evaluate_polynomial_in_evaluation_form and
    compute_kzg_proof_impl's quotient, for a domain of size n."""
    roots = [pow(w, int(format(i, f"0{n.bit_length() - 1}b")[::-1], 2), R) for i in range(n)]
    if z in roots:
        y = evals_brp[roots.index(z)]
    else:
        s = sum(evals_brp[i] * roots[i] * pow(z - roots[i], R - 2, R) for i in range(n))
        y = s * (pow(z, n, R) - 1) * pow(n, R - 2, R) % R
    q = []
    for i in range(n):
        if roots[i] == z:
            acc = 0
            for k in range(n):
                if roots[k] == z:
                    continue
                acc += (evals_brp[k] - y) * roots[k] * pow(z * (z - roots[k]) % R, R - 2, R)
            q.append(acc % R)
        else:
            q.append((evals_brp[i] - y) * pow(roots[i] - z, R - 2, R) % R)
    return y, q, roots


def coeff_form(evals_brp, z, n, w):
    """Interpolate (naively), then Horner and synthetic division."""
    roots = [pow(w, int(format(i, f"0{n.bit_length() - 1}b")[::-1], 2), R) for i in range(n)]
    # coefficients c_k = n^-1 sum_j p(w^j) w^(-jk)
    nat = [0] * n
    for i in range(n):
        nat[int(format(i, f"0{n.bit_length() - 1}b")[::-1], 2)] = evals_brp[i]
    winv = pow(w, R - 2, R)
    ninv = pow(n, R - 2, R)
    c = [sum(nat[j] * pow(winv, j * k, R) for j in range(n)) * ninv % R for k in range(n)]
    acc = c[-1]
    q = [0] * (n - 1)
    for k in range(n - 1, 0, -1):
        q[k - 1] = acc
        acc = (c[k - 1] + z * acc) % R
    return acc, q, roots


def test_evaluation_form_formulas_match_coefficient_form():
    rng = random.Random(4)
    n = 16
    w = pow(7, (R - 1) // n, R)
    for trial in range(6):
        ev = [rng.randrange(R) for _ in range(n)]
        roots = [pow(w, i, R) for i in range(n)]
        z = roots[rng.randrange(n)] if trial % 2 else rng.randrange(R)
        y1, q_eval, dom = spec_eval_form(ev, z, n, w)
        y2, q_coef, _ = coeff_form(ev, z, n, w)
        assert y1 == y2
        for i in range(n):  # the quotient polynomial agrees at every domain point
            v = 0
            for k in reversed(q_coef):
                v = (v * dom[i] + k) % R
            assert v == q_eval[i], (trial, i)


def test_oracle_y_matches_direct_evaluation():
    blob = B.rand_blob(1)
    evals = [int.from_bytes(blob[32 * i:32 * i + 32], "big") for i in range(B.N)]
    # direct interpolation at one point via the barycentric formula in Python
    z = 0x1234567890ABCDEF1234567890ABCDEF % R
    roots = [B.domain_point(i) for i in range(B.N)]
    s = sum(evals[i] * roots[i] * pow(z - roots[i], R - 2, R) for i in range(B.N)) % R
    y = s * (pow(z, B.N, R) - 1) * pow(B.N, R - 2, R) % R
    srs = bytes(96 * B.N)  # the proof point is not checked here
    rc, _, yb = O.kzg_blob_proof(blob, z.to_bytes(32, "big"), srs)
    assert rc == 0 and int.from_bytes(yb, "big") == y
    # a domain point returns the blob element itself
    rc, _, yb = O.kzg_blob_proof(blob, roots[77].to_bytes(32, "big"), srs)
    assert rc == 0 and int.from_bytes(yb, "big") == evals[77]


def test_oracle_rejects_out_of_range():
    blob = bytearray(B.rand_blob(2))
    srs = bytes(96 * B.N)
    assert O.kzg_blob_proof(bytes(blob), R.to_bytes(32, "big"), srs)[0] == -1
    blob[32 * 5:32 * 6] = R.to_bytes(32, "big")
    assert O.kzg_blob_commit(bytes(blob), srs)[0] == -1
    # the zero blob commits to infinity
    assert O.kzg_blob_commit(bytes(32 * B.N), srs) == (0, b"\xc0" + bytes(47))
