"""CPU oracle checks (no GPU).

The oracle (oracle/ssp_oracle.c) is pinned here against independent implementations and against the
expectations the reference's own tests encode (tenchd/spec_spars src/tests.rs):
  * Philox4x64-10 against numpy.random.Philox (an independent implementation of the generator),
  * assembly against scipy.sparse, sketch against a dense numpy product,
  * the factorization against a pure-Python sequential restatement and by unbiasedness E[LDL^T] = L,
  * PCG against a dense pseudo-inverse, and the sampling KATs of tests.rs:215-317,636-667.
"""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.csgraph as csg

from conftest import rand_graph

M64 = (1 << 64) - 1


def py_philox(ctr, key):
    c = list(ctr)
    k = list(key)
    for r in range(10):
        if r:
            k[0] = (k[0] + 0x9E3779B97F4A7C15) & M64
            k[1] = (k[1] + 0xBB67AE8584CAA73B) & M64
        p0 = 0xD2E7470EE14C6C93 * c[0]
        p1 = 0xCA5A826395121157 * c[2]
        c = [(p1 >> 64) ^ c[1] ^ k[0], p1 & M64, (p0 >> 64) ^ c[3] ^ k[1], p0 & M64]
    return c


@pytest.mark.parametrize("key,ctr", [((0, 0), (0, 0, 0, 0)), ((5, 7), (10, 20, 30, 40)),
                                     ((M64, 3), (M64, 1, M64, 2)), ((123456789, 0x5349474e), (77, 3, 0, 0))])
def test_philox_matches_numpy(ora, key, ctr):
    # numpy's Philox increments its 256-bit counter before producing a block
    c = sum(int(x) << (64 * i) for i, x in enumerate(ctr))
    c = (c - 1) % (1 << 256)
    before = [(c >> (64 * i)) & M64 for i in range(4)]
    bg = np.random.Philox(key=np.array(key, dtype=np.uint64), counter=np.array(before, dtype=np.uint64))
    ref = [int(x) for x in bg.random_raw(4)]
    assert [int(x) for x in ora.philox4x64(ctr, *key)] == ref
    assert py_philox(ctr, key) == ref


def test_sketch_entry_bit_layout(ora):
    seed = 11
    for e in (0, 1, 12345):
        for j in (0, 1, 63, 64, 200, 255, 256, 1000):
            w = py_philox((e, j >> 8, 0, 0), (seed, 0x5349474e))[(j >> 6) & 3]
            want = -1.0 if (w >> (j & 63)) & 1 else 1.0
            assert ora.sketch_entry(seed, 0, e, j) == want
            w = py_philox((e, j >> 3, 0, 0), (seed, 0x554e4946))[(j >> 1) & 3]
            x = (w >> 32) if (j & 1) else (w & 0xFFFFFFFF)
            assert ora.sketch_entry(seed, 1, e, j) == 2.0 * ((x + 0.5) / 4294967296.0) - 1.0
    vals = np.array([ora.sketch_entry(3, 0, e, j) for e in range(64) for j in range(64)])
    assert abs(vals.mean()) < 0.05


def test_coins_and_factor_uniforms_layout(ora):
    for e in (0, 1, 5, 1023):
        w = py_philox((e >> 2, 0, 0, 0), (9, 0x434f494e))[e & 3]
        assert ora.coin(9, e) == (w >> 11) * 2.0 ** -53
    c = ora.coins(4, 20000)
    assert 0.0 <= c.min() and c.max() < 1.0 and abs(c.mean() - 0.5) < 0.01


def _edges_ref(A):
    U = sp.triu(A, 1).tocsc()
    U.sort_indices()
    rows = U.indices.astype(np.int32)
    cols = np.repeat(np.arange(A.shape[0]), np.diff(U.indptr)).astype(np.int32)
    return rows, cols, U.data


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_edges_and_laplacian_vs_scipy(ora, seed):
    A = rand_graph(300, 1200, seed)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    r1, r2, rw = _edges_ref(A)
    assert np.array_equal(v1, r1) and np.array_equal(v2, r2) and np.array_equal(w, rw)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    L = sp.csc_matrix((va, ri, cp), shape=(n, n))
    deg = np.asarray(A.sum(axis=0)).ravel()
    Lref = sp.diags(deg) - A
    assert abs(L - Lref).max() < 1e-12
    # off-diagonals exactly -w; column sums ~0 and symmetry (check_diagonal, sparsifier.rs:806-817)
    assert np.abs(np.asarray(L.sum(axis=0))).max() <= 1e-10
    assert abs(L - L.T).max() == 0.0
    # diagonal accumulated in edge order
    d = np.zeros(n)
    for a, b, x in zip(v1, v2, w):
        d[a] += x
        d[b] += x
    assert np.array_equal(L.diagonal(), d)


def test_edge_extraction_rejects_bad_input(ora):
    A = rand_graph(50, 100, 3)
    bad = A.copy()
    bad.data = -bad.data
    with pytest.raises(ValueError):
        ora.extract_edges(50, bad.indptr, bad.indices, bad.data)
    idx = A.indices.copy()
    s, e = A.indptr[5], A.indptr[6]
    if e - s >= 2:
        idx[s], idx[s + 1] = idx[s + 1], idx[s]
        with pytest.raises(ValueError):
            ora.extract_edges(50, A.indptr, idx, A.data)


def test_zero_weights_and_lower_triangle_ignored(ora):
    # only row < col with value != 0 become edges (stream.rs:46, sparsifier.rs:365)
    A = sp.csc_matrix(np.array([[5.0, 0.0, 2.0], [1.0, 3.0, 0.0], [0.0, 4.0, 0.0]]))
    A.data[A.data == 0] = 0
    v1, v2, w = ora.extract_edges(3, A.indptr, A.indices, A.data)
    assert list(zip(v1, v2, w)) == [(0, 2, 2.0)]


@pytest.mark.parametrize("uniform", [False, True])
def test_sketch_vs_dense_product(ora, uniform):
    A = rand_graph(120, 500, 7)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    k, scale, seed = 40, 1.7, 5
    Y = ora.sketch(n, v1, v2, w, k, scale, seed, uniform)
    m = len(v1)
    Q = np.array([[ora.sketch_entry(seed, int(uniform), e, j) * scale for j in range(k)] for e in range(m)])
    B = np.zeros((m, n))
    B[np.arange(m), v1] = -np.sqrt(w)
    B[np.arange(m), v2] = np.sqrt(w)
    assert np.abs(Y - B.T @ Q).max() < 1e-12
    # jl_sketch_zero (tests.rs:481-511): every column sums to ~0
    assert np.abs(Y.sum(axis=0)).max() < 1e-10
    # exact: sequential accumulation in edge order
    Yx = np.zeros((n, k))
    for e in range(m):
        for v, b in ((v1[e], -math.sqrt(w[e])), (v2[e], math.sqrt(w[e]))):
            for j in range(k):
                Yx[v, j] = Yx[v, j] + Q[e, j] * b
    assert np.array_equal(Y, Yx)


# ---------------------------------------------------------------- factorization
def _chunk_scan(a):
    c = [0.0] * len(a)
    carry = 0.0
    for base in range(0, len(a), 32):
        ln = min(32, len(a) - base)
        t = [a[base + l] if l < ln else 0.0 for l in range(32)]
        s = 1
        while s < 32:
            t = [t[l - s] + t[l] if l >= s else t[l] for l in range(32)]
            s <<= 1
        for l in range(ln):
            c[base + l] = carry + t[l] if base > 0 else t[l]
        carry = c[base + ln - 1]
    return c


def py_factor(n, cp, ri, va, seed, ora):
    """Sequential approximate Cholesky in (priority, id) order -- the specification the
    level-parallel oracle and the CUDA kernels must reproduce bit for bit."""
    bags = [[] for _ in range(n)]
    for c in range(n):
        for p in range(cp[c], cp[c + 1]):
            r = ri[p]
            if r > c and abs(va[p]) != 0.0:
                bags[c].append((int(r), abs(float(va[p]))))
                bags[r].append((c, abs(float(va[p]))))
    prio = [ora.priority(seed, v) for v in range(n)]
    order = sorted(range(n), key=lambda v: (prio[v], v))
    dead = [False] * n
    cols = {}
    D = [0.0] * n
    for v in order:
        E = sorted((u, w) for (u, w) in bags[v] if not dead[u])
        merged = []
        for u, w in E:
            if merged and merged[-1][0] == u:
                merged[-1][1] = merged[-1][1] + w
            else:
                merged.append([u, w])
        merged.sort(key=lambda t: (t[1], t[0]))
        cnt = len(merged)
        dead[v] = True
        if cnt == 0:
            cols[v] = []
            continue
        c = _chunk_scan([w for _, w in merged])
        S = c[-1]
        for i in range(cnt - 1):
            rem = S - c[i]
            tgt = ora.lib().ora_factor_uniform(seed, v, i) * rem
            lo, hi = i + 1, cnt
            while lo < hi:
                mid = (lo + hi) // 2
                if (c[mid] - c[i]) < tgt:
                    lo = mid + 1
                else:
                    hi = mid
            j = min(lo, cnt - 1)
            a, b = max(merged[i][0], merged[j][0]), min(merged[i][0], merged[j][0])
            wf = (merged[i][1] * rem) / S
            bags[a].append((b, wf))
            bags[b].append((a, wf))
        cols[v] = [(u, -(w / S)) for u, w in merged]
        D[v] = S
    return cols, D


def _canon(F, n):
    out = {}
    for v in range(n):
        ent = sorted(zip(F.rows[F.colstart[v]:F.colstart[v + 1]].tolist(),
                         F.vals[F.colstart[v]:F.colstart[v + 1]].tolist()))
        out[v] = ent
    return out


@pytest.mark.parametrize("seed", [0, 3])
def test_factor_level_parallel_equals_sequential(ora, seed):
    A = rand_graph(150, 450, seed + 10)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    F = ora.Factor(n, cp, ri, va, seed, 0)
    cols, D = py_factor(n, cp, ri, va, seed, ora)
    got = _canon(F, n)
    for v in range(n):
        assert got[v] == sorted(cols[v]), v
    assert F.D.tolist() == D
    # level structure: every entry (row r of column v) is eliminated at a later level
    for v in range(n):
        for p in range(F.colstart[v], F.colstart[v + 1]):
            assert F.level[F.rows[p]] > F.level[v]


def test_factor_dense_tail_structure(ora):
    A = rand_graph(200, 900, 42)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    F = ora.Factor(n, cp, ri, va, 1, 60)
    assert 0 < F.dense_start < n and n - F.dense_start <= 60
    lv = F.level[F.order[F.dense_start:]]
    assert np.array_equal(lv, np.arange(lv[0], lv[0] + len(lv)))  # one vertex per level
    for v in range(n):
        for p in range(F.colstart[v], F.colstart[v + 1]):
            assert F.level[F.rows[p]] > F.level[v]
    # connected graph: exactly one zero pivot (the last vertex)
    ncomp = csg.connected_components(A, directed=False)[0]
    assert int((F.D == 0).sum()) == ncomp


@pytest.mark.parametrize("dense", [0, 40])
def test_factor_unbiased(ora, dense):
    """Approximate Cholesky is an unbiased estimator: E[L D L^T] = L_G."""
    A = rand_graph(60, 200, 5)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    Lg = sp.csc_matrix((va, ri, cp), shape=(n, n)).toarray()
    errs = []
    acc = np.zeros((n, n))
    S = 0
    for s in range(1, 801):
        F = ora.Factor(n, cp, ri, va, s, dense)
        Ld = F.dense_L()
        acc += Ld @ np.diag(F.D) @ Ld.T
        S += 1
        if s in (50, 800):
            errs.append(np.abs(acc / S - Lg).max() / np.abs(Lg).max())
    assert errs[1] < errs[0] and errs[1] < 0.02


@pytest.mark.parametrize("maxdeg", [16, 24])
def test_factor_truncation(ora, maxdeg):
    """Truncated elimination: every vertex left once the Schur complement's average degree exceeds
    maxdeg sits in one final level with no L entries and D = its merged live weight sum; the
    preconditioner stays SPD and PCG still converges to the same solution."""
    A = rand_graph(400, 2400, 21)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    F = ora.Factor(n, cp, ri, va, 3, 0, maxdeg)
    last = F.level == F.level.max()
    assert 0 < last.sum() < n
    assert np.all(np.diff(F.colstart)[last] == 0) and np.all(F.D[last] > 0)
    Ffull = ora.Factor(n, cp, ri, va, 3, 0, 0)
    # eliminated vertices are identical to the untruncated run (same order, same columns)
    elim = ~last
    assert np.array_equal(F.D[elim], Ffull.D[elim])
    Y = ora.sketch(n, v1, v2, w, 6, 1 / math.sqrt(6), 1)
    Z, it, rel, rc = ora.pcg(n, cp, ri, va, F, Y, 1e-10, 0.0, 400)
    Zf, itf, relf, rcf = ora.pcg(n, cp, ri, va, Ffull, Y, 1e-10, 0.0, 400)
    assert rc == 0 and rel.max() < 1e-9
    dz, df = Z[v1] - Z[v2], Zf[v1] - Zf[v2]
    assert np.abs(dz - df).max() <= 1e-7 * np.abs(df).max()


def test_precond_is_spd_on_range(ora):
    A = rand_graph(80, 300, 8)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    F = ora.Factor(n, cp, ri, va, 2, 0)
    M = np.column_stack([F.precond(np.eye(n)[:, i]) for i in range(n)])
    Ld = F.dense_L()
    Dp = np.diag([1 / d if d != 0 else 1.0 for d in F.D])
    assert np.abs(M - np.linalg.inv(Ld.T) @ Dp @ np.linalg.inv(Ld)).max() < 1e-9
    assert np.abs(M - M.T).max() < 1e-9


@pytest.mark.parametrize("dense", [0, 30])
def test_pcg_matches_pseudoinverse(ora, dense):
    A = rand_graph(200, 800, 9)
    n = A.shape[0]
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    F = ora.Factor(n, cp, ri, va, 0, dense)
    Y = ora.sketch(n, v1, v2, w, 12, 1 / math.sqrt(12), 0)
    Z, it, rel, rc = ora.pcg(n, cp, ri, va, F, Y, 1e-11, 0.0, 400)
    assert rc == 0 and rel.max() < 1e-9
    Lg = sp.csc_matrix((va, ri, cp), shape=(n, n)).toarray()
    Zx = np.linalg.pinv(Lg) @ (Y - Y.mean(0))
    # compare what the leverage estimate uses: differences across edges (per-component nullspace drops out)
    dz, dx = Z[v1] - Z[v2], Zx[v1] - Zx[v2]
    assert np.abs(dz - dx).max() <= 1e-8 * np.abs(dx).max()
    assert it.max() < 100


def test_diff_norms_and_probs(ora):
    rng = np.random.default_rng(1)
    Z = rng.standard_normal((50, 77))
    v1 = rng.integers(0, 50, 200).astype(np.int32)
    v2 = rng.integers(0, 50, 200).astype(np.int32)
    d = ora.diff_norms(v1, v2, Z)
    assert np.allclose(d, np.sqrt(((Z[v1] - Z[v2]) ** 2).sum(1)), rtol=1e-14, atol=0)
    w = rng.uniform(0.5, 2, 200)
    beta, k = 147.3, 54.0
    p = ora.probs(w, d, beta, k)
    # reference expression: (beta * -1 * value * d.powi(2) / k).min(1.0) with value = -w
    ref = np.array([min((((beta * -1.0) * -wi) * (di * di)) / k, 1.0) for wi, di in zip(w, d)])
    assert np.array_equal(p, ref)
    assert (p >= 0).all() and (p <= 1).all()


# ---------------------------------------------------------------- sampling KATs (tests.rs)
def test_sampling_verify_ratios(ora, ssp):
    """tests.rs:215-261: with p = 0.5, about half the edges survive and the degree sum drops by sqrt(2)
    (kept edges are reweighted by w/sqrt(p))."""
    G = ssp.gen_grid2d(150, 150)
    n = G.n
    v1, v2, w = ora.extract_edges(n, G.colptr, G.rowidx, G.values)
    lg = ora.laplacian(n, v1, v2, w)
    for seed in range(3):
        coins = ora.coins(seed, len(v1))
        (hcp, hri, hva), keep = ora.sample_apply(n, v1, v2, w, np.full(len(v1), 0.5), coins, 0, lg)
        H = sp.csc_matrix((hva, hri, hcp), shape=(n, n))
        after = (H.nnz - np.count_nonzero(H.diagonal())) // 2
        assert after == keep.sum()
        assert abs(len(v1) / after - 2.0) <= 0.05
        before_diag = lg[2][lg[1] == np.repeat(np.arange(n), np.diff(lg[0]))].sum()
        assert abs(before_diag / H.diagonal().sum() - 2.0 / math.sqrt(2.0)) <= 0.05
        # check_diagonal after sampling: columns still sum to ~0
        assert np.abs(np.asarray(H.sum(axis=0))).max() <= 1e-10
        # E(H) is a subset of E(G) (check_for_additions, tests.rs:636-667)
        Hs = sp.triu(H, 1) != 0
        Gs = sp.triu(sp.csc_matrix((lg[2], lg[1], lg[0]), shape=(n, n)), 1) != 0
        assert (Hs > Gs).nnz == 0


def test_sampling_forced_components(ora):
    """tests.rs:267-317: a 100-node path plus 10 shortcuts; deleting every second path edge of each
    block of ten (p = 0) while keeping the rest (p = 1) leaves exactly 40 connected components."""
    edges = [(i, i + 1) for i in range(99)] + [(10 * i, 10 * i + 9) for i in range(10)]
    n = 100
    A = sp.coo_matrix((np.ones(len(edges)), tuple(np.array(edges).T)), shape=(n, n))
    A = (A + A.T).tocsc()
    A.sort_indices()
    v1, v2, w = ora.extract_edges(n, A.indptr, A.indices, A.data)
    lg = ora.laplacian(n, v1, v2, w)
    p = np.ones(len(v1))
    for i in range(10):
        for j in range(5):
            idx = i * 11 + 2 + 2 * j
            if idx == len(v1):
                break
            p[idx] = 0.0
    coins = ora.coins(0, len(v1))
    (hcp, hri, hva), keep = ora.sample_apply(n, v1, v2, w, p, coins, 0, lg)
    H = sp.csc_matrix((hva, hri, hcp), shape=(n, n))
    Hadj = sp.triu(H, 1) != 0
    assert csg.connected_components(A, directed=False)[0] == 1
    assert csg.connected_components(Hadj, directed=False)[0] == 40
    assert np.array_equal(keep, p == 1.0)


def test_reweight_inv_p_unbiased(ora, ssp):
    G = ssp.gen_grid2d(60, 60)
    n = G.n
    v1, v2, w = ora.extract_edges(n, G.colptr, G.rowidx, G.values)
    lg = ora.laplacian(n, v1, v2, w)
    tot = 0.0
    for seed in range(20):
        coins = ora.coins(seed, len(v1))
        (hcp, hri, hva), _ = ora.sample_apply(n, v1, v2, w, np.full(len(v1), 0.25), coins, 1, lg)
        H = sp.csc_matrix((hva, hri, hcp), shape=(n, n))
        tot += H.diagonal().sum()
    assert abs(tot / 20 / (2 * w.sum()) - 1.0) < 0.02


def test_oracle_er_generator_is_the_library_generator(ora, ssp):
    # the CPU baselines build their ER samples with the oracle's generator (no library in the reference
    # process); it must give the library's graph edge for edge
    for n, deg, seed in [(2, 20.0, 3), (50, 9.0, 9), (5000, 20.0, 1), (60_000, 20.0, 11)]:
        G = ssp.gen_er(n, deg, 0.5, 2.0, seed)
        a = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
        b = ora.gen_er(n, deg, 0.5, 2.0, seed)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
