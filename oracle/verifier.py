"""Verifier of wide-Fibonacci proofs (JSON wire), a Python restatement of the reference's
verifier: src/examples/wide_fibonacci.zig:360-433 (verify), src/core/verifier.zig (OODS check),
src/core/pcs/verifier.zig:79-178 (verifyValues), src/core/fri.zig (FRI), src/core/vcs_lifted/
verifier.zig (lifted Merkle), src/core/pcs/quotients/fri_answers.zig (quotient answers).

TEST INFRASTRUCTURE ONLY (the oracle's self-check): imported by tests/ and by the CPU legs of
bench.py. It raises VerificationError on the first failed check.
"""
from __future__ import annotations

import hashlib
import json
import struct

P = (1 << 31) - 1


class VerificationError(Exception):
    pass


# ---------------------------------------------------------------------------
# Fields (src/core/fields/{m31,cm31,qm31}.zig)
# ---------------------------------------------------------------------------
def cmul(x, y):
    return ((x[0] * y[0] - x[1] * y[1]) % P, (x[0] * y[1] + x[1] * y[0]) % P)


def cadd(x, y):
    return ((x[0] + y[0]) % P, (x[1] + y[1]) % P)


def csub(x, y):
    return ((x[0] - y[0]) % P, (x[1] - y[1]) % P)


def cinv(x):
    d = pow((x[0] * x[0] + x[1] * x[1]) % P, P - 2, P)
    return (x[0] * d % P, (-x[1]) * d % P)


def q(a, b=0, c=0, d=0):
    return ((a % P, b % P), (c % P, d % P))


def qadd(x, y):
    return (cadd(x[0], y[0]), cadd(x[1], y[1]))


def qsub(x, y):
    return (csub(x[0], y[0]), csub(x[1], y[1]))


def mul_r(x):  # x * (2 + i)
    return ((2 * x[0] - x[1]) % P, (x[0] + 2 * x[1]) % P)


def qmul(x, y):
    ac = cmul(x[0], y[0])
    bd = cmul(x[1], y[1])
    cross = csub(csub(cmul(cadd(x[0], x[1]), cadd(y[0], y[1])), ac), bd)
    return (cadd(ac, mul_r(bd)), cross)


def qmulm(x, m):
    return ((x[0][0] * m % P, x[0][1] * m % P), (x[1][0] * m % P, x[1][1] * m % P))


def qmulc(x, c):
    return (cmul(x[0], c), cmul(x[1], c))


def qconj(x):
    return (x[0], ((-x[1][0]) % P, (-x[1][1]) % P))


def qinv(x):
    denom = csub(cmul(x[0], x[0]), mul_r(cmul(x[1], x[1])))
    di = cinv(denom)
    return (cmul(x[0], di), cmul(((-x[1][0]) % P, (-x[1][1]) % P), di))


def qflat(x):
    return [x[0][0], x[0][1], x[1][0], x[1][1]]


def qfrom(lst):
    return ((lst[0], lst[1]), (lst[2], lst[3]))


# ---------------------------------------------------------------------------
# Circle group (src/core/circle.zig)
# ---------------------------------------------------------------------------
def mpadd(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


_GEN = (2, 1268011823)
_DOUBLES = []
_cur = _GEN
for _ in range(31):
    _DOUBLES.append(_cur)
    _cur = mpadd(_cur, _cur)


def index_point(idx):
    idx &= (1 << 31) - 1
    acc = (1, 0)
    b = 0
    while idx:
        if idx & 1:
            acc = mpadd(acc, _DOUBLES[b])
        idx >>= 1
        b += 1
    return acc


def subgroup_gen(log):
    return 1 << (31 - log)


def half_odds(log):
    return (subgroup_gen(log + 2), subgroup_gen(log), log)  # (initial, step, log)


def coset_index(c, i):
    return (c[0] + c[1] * i) & ((1 << 31) - 1)


def domain_index(log, i):
    """CanonicCoset(log).circleDomain().indexAt(i)."""
    half = half_odds(log - 1)
    hs = 1 << (log - 1)
    if i < hs:
        return coset_index(half, i)
    return (-coset_index(half, i - hs)) & ((1 << 31) - 1)


def bitrev(i, log):
    r = 0
    for _ in range(log):
        r = (r << 1) | (i & 1)
        i >>= 1
    return r


def qpadd(a, b):
    return (qsub(qmul(a[0], b[0]), qmul(a[1], b[1])), qadd(qmul(a[0], b[1]), qmul(a[1], b[0])))


def qdouble_x(x):
    s = qmul(x, x)
    return qsub(qadd(s, s), q(1))


# ---------------------------------------------------------------------------
# Channel (src/core/channel/blake2s.zig), Merkle hasher (src/core/vcs_lifted/blake2_merkle.zig)
# ---------------------------------------------------------------------------
def b2s(data: bytes) -> bytes:
    return hashlib.blake2s(data).digest()


LEAF = b"leaf" + b"\0" * 60
NODE = b"node" + b"\0" * 60


class Channel:
    def __init__(self):
        self.digest = b"\0" * 32
        self.n_draws = 0

    def _set(self, d):
        self.digest, self.n_draws = d, 0

    def mix_felts(self, felts):
        self._set(b2s(self.digest + b"".join(struct.pack("<4I", *qflat(f)) for f in felts)))

    def mix_u32s(self, words):
        self._set(b2s(self.digest + struct.pack(f"<{len(words)}I", *words)))

    def mix_u64(self, v):
        self.mix_u32s([v & 0xFFFFFFFF, v >> 32])

    def mix_root(self, root: bytes):
        self._set(b2s(self.digest + root))

    def draw_u32s(self):
        h = b2s(self.digest + struct.pack("<I", self.n_draws) + b"\0")
        self.n_draws += 1
        return list(struct.unpack("<8I", h))

    def draw_secure_felt(self):
        while True:
            w = self.draw_u32s()
            if all(x < 2 * P for x in w):
                return q(*(x % P for x in w[:4]))


def pow_ok(digest: bytes, bits: int, nonce: int) -> bool:
    prefix = b2s(struct.pack("<I", 0x12345678) + b"\0" * 12 + digest + struct.pack("<I", bits))
    h = b2s(prefix + struct.pack("<Q", nonce))
    v = int.from_bytes(h[:16], "little")
    tz = 128 if v == 0 else (v & -v).bit_length() - 1
    return tz >= bits


def merkle_verify(root, max_log, positions, columns, witness, col_logs=None):
    """Lifted Merkle verification (src/core/vcs_lifted/verifier.zig:94-250). positions: queried leaf
    indices (any order, duplicates allowed); columns[c][j] value of column c at positions[j] (for a
    column smaller than the tree, its value at the lifted index). A leaf hashes the row of values in
    column order stably sorted by log size (col_logs; equal sizes when omitted)."""
    if not columns:
        if witness:
            raise VerificationError("witness for an empty tree")
        return
    corder = sorted(range(len(columns)), key=lambda c: ((col_logs[c] if col_logs else 0), c))
    order = sorted(range(len(positions)), key=lambda j: (positions[j], j))
    leaves = {}
    for j in order:
        pos = positions[j]
        row = b"".join(struct.pack("<I", columns[c][j]) for c in corder)
        h = b2s(LEAF + row)
        if pos in leaves and leaves[pos] != h:
            raise VerificationError("duplicate query mismatch")
        leaves[pos] = h
    prev = sorted(leaves.items())
    wi = 0
    for _ in range(max_log):
        cur = []
        p = 0
        while p < len(prev):
            idx, h = prev[p]
            if p + 1 < len(prev) and prev[p + 1][0] == idx ^ 1:
                left, right, step = h, prev[p + 1][1], 2
            else:
                if wi >= len(witness):
                    raise VerificationError("witness too short")
                w = witness[wi]
                wi += 1
                left, right = (h, w) if idx & 1 == 0 else (w, h)
                step = 1
            cur.append((idx >> 1, b2s(NODE + left + right)))
            p += step
        prev = cur
    if wi != len(witness):
        raise VerificationError("witness too long")
    if len(prev) != 1 or prev[0][1] != root:
        raise VerificationError("root mismatch")


def coset_vanishing_q(coset_log, initial_idx, step_idx, p):
    ini = index_point(initial_idx)
    hs = index_point(step_idx // 2)
    qp = qpadd(qpadd(p, (q(ini[0]), q(-ini[1]))), (q(hs[0]), q(hs[1])))
    x = qp[0]
    for _ in range(1, coset_log):
        x = qdouble_x(x)
    return x


def verify_wide_fib(proof_bytes: bytes, log_n_rows: int, sequence_len: int, channel_seed: int | None = None):
    pr = json.loads(proof_bytes)
    cfg = pr["config"]
    fc = cfg["fri_config"]
    pow_bits, B, log_last, n_queries = cfg["pow_bits"], fc["log_blowup_factor"], fc["log_last_layer_degree_bound"], \
        fc["n_queries"]
    if fc.get("fold_step", 1) != 1 or cfg.get("lifting_log_size") is not None:
        raise VerificationError("unsupported config")
    n, W = log_n_rows, sequence_len
    roots = [bytes(c) for c in pr["commitments"]]
    if len(roots) != 3:
        raise VerificationError("expected 3 commitments")
    ch = Channel()
    ch.mix_felts([q(pow_bits, B, n_queries, log_last)])
    ch.mix_root(roots[0])
    ch.mix_root(roots[1])
    ch.mix_u32s([n, W])
    if channel_seed is not None:
        ch.mix_u64(channel_seed)
    random_coeff = ch.draw_secure_felt()
    ch.mix_root(roots[2])
    t = ch.draw_secure_felt()
    t2 = qmul(t, t)
    inv = qinv(qadd(t2, q(1)))
    oods = (qmul(qsub(q(1), t2), inv), qmul(qadd(t, t), inv))

    sv = pr["sampled_values"]
    if len(sv) != 3 or len(sv[0]) != 0 or len(sv[1]) != W or len(sv[2]) != 8:
        raise VerificationError("sampled values shape")
    main = [qfrom(c[0]) for c in sv[1]]
    comp = [qfrom(c[0]) for c in sv[2]]
    # composition OODS check (src/core/proof.zig:37-69, src/core/verifier.zig:96-110)
    basis = [q(1), q(0, 1), q(0, 0, 1), q(0, 0, 0, 1)]
    left, right = q(0), q(0)
    for k in range(4):
        left = qadd(left, qmul(comp[k], basis[k]))
        right = qadd(right, qmul(comp[4 + k], basis[k]))
    pt = oods
    for _ in range(n + 1 - 2):
        pt = qpadd(pt, pt)
    comp_eval = qadd(left, qmul(pt[0], right))
    dinv = qinv(coset_vanishing_q(n, subgroup_gen(n + 1), subgroup_gen(n), oods))
    acc = q(0)
    a, b = main[0], main[1]
    for k in range(2, W):
        c = main[k]
        acc = qadd(qmul(acc, random_coeff), qmul(qsub(c, qadd(qmul(a, a), qmul(b, b))), dinv))
        a, b = b, c
    if acc != comp_eval:
        raise VerificationError("OODS mismatch")

    ch.mix_felts(main + comp)
    quot_coeff = ch.draw_secure_felt()
    # one batch at the OODS point: every column's sample, powers 1, q, q^2, ... in column order
    rp = q(1)
    entries = []
    for c, v in enumerate(main + comp):
        entries.append((c, v, rp))
        rp = qmul(rp, quot_coeff)
    return _verify_pcs_tail(pr, ch, roots, [0, W, 8], [(oods, entries)], n + B, B, pow_bits, log_last, n_queries)


def _verify_pcs_tail(pr, ch, roots, tree_cols, batches, L, B, pow_bits, log_last, n_queries, tree_logs=None):
    """FRI commitments and alphas, last layer, proof of work, queries, the trees' Merkle
    decommitments and the FRI decommitment, for a proof whose trees hold tree_cols[t] columns on
    the lifting domain of log size L. tree_logs[t] (optional): the committed log sizes of tree t's
    columns; a tree's depth is its largest column, and the preprocessed tree (tree 0), when smaller
    than L, is queried at the positions mapped down (src/core/pcs/utils.zig:292-314). batches:
    [(point, [(flat column, value, random power)])] (src/core/pcs/quotients/fri_answers.zig,
    src/core/fri.zig)."""
    fri = pr["fri_proof"]
    ch.mix_root(bytes(fri["first_layer"]["commitment"]))
    alphas = [ch.draw_secure_felt()]
    n_inner = (L - 1) - (log_last + B)
    if len(fri["inner_layers"]) != n_inner:
        raise VerificationError("number of FRI layers")
    for layer in fri["inner_layers"]:
        ch.mix_root(bytes(layer["commitment"]))
        alphas.append(ch.draw_secure_felt())
    last = [qfrom(v) for v in fri["last_layer_poly"]]
    if len(last) > (1 << log_last):
        raise VerificationError("last layer degree")
    ch.mix_felts(last)
    nonce = pr["proof_of_work"]
    if not pow_ok(ch.digest, pow_bits, nonce):
        raise VerificationError("proof of work")
    ch.mix_u64(nonce)
    queries = []
    mask = (1 << L) - 1
    while len(queries) < n_queries:
        for x in ch.draw_u32s():
            queries.append(x & mask)
            if len(queries) == n_queries:
                break
    queries = sorted(set(queries))

    qv = pr["queried_values"]
    dec = pr["decommitments"]
    if len(qv) != len(tree_cols) or len(dec) != len(tree_cols):
        raise VerificationError("number of trees")
    cols = []
    for t_idx, ncols in enumerate(tree_cols):
        tcols = qv[t_idx]
        if len(tcols) != ncols or any(len(c) != len(queries) for c in tcols):
            raise VerificationError("queried values shape")
        if ncols == 0:
            if dec[t_idx]["hash_witness"]:
                raise VerificationError("preprocessed tree shape")
            continue
        logs = tree_logs[t_idx] if tree_logs else None
        depth = max(logs) if logs else L
        positions = queries
        if depth != L:
            if t_idx != 0 or depth > L:
                raise VerificationError("tree size")
            sh = L - depth + 1
            positions = [((p >> sh) << 1) + (p & 1) for p in queries]
        merkle_verify(roots[t_idx], depth, positions, tcols, [bytes(h) for h in dec[t_idx]["hash_witness"]], logs)
        cols.extend(tcols)

    # quotient answers at the queries (src/core/pcs/quotients/fri_answers.zig, row_evaluation.zig)
    consts = []
    for point, entries in batches:
        cy = qsub(qconj(point[1]), point[1])
        sum_a, sum_b, lc = q(0), q(0), []
        for c, v, rp in entries:
            aa = qsub(qconj(v), v)
            bb = qsub(qmul(v, cy), qmul(aa, point[1]))
            lc.append((c, qmul(rp, cy)))
            sum_a = qadd(sum_a, qmul(rp, aa))
            sum_b = qadd(sum_b, qmul(rp, bb))
        consts.append((point, lc, sum_a, sum_b))
    answers = []
    for j, pos in enumerate(queries):
        x, y = index_point(domain_index(L, bitrev(pos, L)))
        acc = q(0)
        for point, lc, sum_a, sum_b in consts:
            num = q(0)
            for c, coef in lc:
                num = qadd(num, qmulm(coef, cols[c][j]))
            num = qsub(num, qadd(qmulm(sum_a, y), sum_b))
            prx, pry, pix, piy = point[0][0], point[1][0], point[0][1], point[1][1]
            den = csub(cmul(csub(prx, (x, 0)), piy), cmul(csub(pry, (y, 0)), pix))
            acc = qadd(acc, qmulc(num, cinv(den)))
        answers.append(acc)

    # FRI decommitment (src/core/fri.zig:171-216, folding.zig:160-230)
    def layer_check(layer, qpos, qevals, log_size, fold):
        witness = [qfrom(w) for w in layer["fri_witness"]]
        wi = 0
        dpos, dvals, folded = [], [], []
        i = 0
        while i < len(qpos):
            key = qpos[i] >> 1
            end = i
            while end < len(qpos) and qpos[end] >> 1 == key:
                end += 1
            sub = []
            at = i
            for pos in (key << 1, (key << 1) + 1):
                dpos.append(pos)
                if at < end and qpos[at] == pos:
                    sub.append(qevals[at])
                    at += 1
                else:
                    if wi >= len(witness):
                        raise VerificationError("fri witness too short")
                    sub.append(witness[wi])
                    wi += 1
            dvals.extend(sub)
            folded.append(fold(key, sub[0], sub[1]))
            i = end
        if wi != len(witness):
            raise VerificationError("fri witness too long")
        colvals = [[qflat(v)[k] for v in dvals] for k in range(4)]
        merkle_verify(bytes(layer["commitment"]), log_size, dpos, colvals,
                      [bytes(h) for h in layer["decommitment"]["hash_witness"]])
        nq = sorted(set(p >> 1 for p in qpos))
        return nq, folded

    def ibfly_fold(f0, f1, inv_t, alpha):
        a = qadd(f0, f1)
        b = qmulm(qsub(f0, f1), inv_t)
        return qadd(a, qmul(alpha, b))

    def circle_fold(key, f0, f1):
        y = index_point(coset_index(half_odds(L - 1), bitrev(key, L - 1)))[1]
        return ibfly_fold(f0, f1, pow(y, P - 2, P), alphas[0])

    qpos, qev = layer_check(fri["first_layer"], queries, answers, L, circle_fold)
    for k, layer in enumerate(fri["inner_layers"]):
        lg = L - 1 - k

        def line_fold(key, f0, f1, lg=lg, alpha=alphas[k + 1]):
            x = index_point(coset_index(half_odds(lg), bitrev(key, lg - 1)))[0]
            return ibfly_fold(f0, f1, pow(x, P - 2, P), alpha)

        qpos, qev = layer_check(layer, qpos, qev, lg, line_fold)
    # last layer: evaluations at the remaining queries equal the last polynomial
    last_log = log_last + B
    dom = half_odds(last_log)
    for pos, ev in zip(qpos, qev):
        x = q(index_point(coset_index(dom, bitrev(pos, last_log)))[0])
        # LinePoly.evalAtPoint: fold over [x, pi(x), ...] (coefficients in bit-reversed order)
        coeffs = list(last)
        lg = len(coeffs).bit_length() - 1
        factors, cur = [], x
        for _ in range(lg):
            factors.append(cur)
            cur = qdouble_x(cur)

        def fold(vals, fs):
            if len(vals) == 1:
                return vals[0]
            h = len(vals) // 2
            return qadd(fold(vals[:h], fs[1:]), qmul(fold(vals[h:], fs[1:]), fs[0]))

        if fold(coeffs, factors) != ev:
            raise VerificationError("last layer evaluation")
    return True


def verify_logup_xor(proof_bytes: bytes, log_n: int, log_table: int = 16, channel_seed: int | None = None):
    """Verifier of the LogUp XOR-lookup AIR proofs of the B200 prover (the AIR is described in
    stwo-zig_b200/csrc/xor_prover.cu; it has no reference counterpart): a main component of 2^log_n
    rows and a table component of 2^log_table rows under the reference's lifted PCS. Checks the
    transcript, the cancellation of the two LogUp claimed sums, both LogUp transition constraints
    and the composition at the OODS point (each component at the point doubled to its size, with
    its own vanishing polynomial), and the PCS / FRI decommitments with lifted trees."""
    pr = json.loads(proof_bytes)
    cfg = pr["config"]
    fc = cfg["fri_config"]
    pow_bits, B, log_last, n_queries = cfg["pow_bits"], fc["log_blowup_factor"], fc["log_last_layer_degree_bound"], \
        fc["n_queries"]
    if fc.get("fold_step", 1) != 1 or cfg.get("lifting_log_size") is not None:
        raise VerificationError("unsupported config")
    if pr["statement"] != {"log_n": log_n, "log_table": log_table}:
        raise VerificationError("statement mismatch")
    n, t = log_n, log_table
    L = max(n, t)
    roots = [bytes(c) for c in pr["commitments"]]
    if len(roots) != 4:
        raise VerificationError("expected 4 commitments")
    ch = Channel()
    ch.mix_felts([q(pow_bits, B, n_queries, log_last)])
    ch.mix_root(roots[0])
    ch.mix_root(roots[1])
    ch.mix_u32s([log_n, log_table])
    if channel_seed is not None:
        ch.mix_u64(channel_seed)
    z = ch.draw_secure_felt()
    alpha = ch.draw_secure_felt()
    alpha2 = qmul(alpha, alpha)
    ch.mix_root(roots[2])
    claimed = [qfrom(c) for c in pr["claimed_sums"]]
    if len(claimed) != 2:
        raise VerificationError("claimed sums")
    ch.mix_felts(claimed)
    if qadd(claimed[0], claimed[1]) != q(0):
        raise VerificationError("LogUp claimed sums do not cancel")
    random_coeff = ch.draw_secure_felt()
    ch.mix_root(roots[3])
    t_ = ch.draw_secure_felt()
    t2 = qmul(t_, t_)
    inv = qinv(qadd(t2, q(1)))
    oods = (qmul(qsub(q(1), t2), inv), qmul(qadd(t_, t_), inv))
    g = index_point(subgroup_gen(L))
    prev = qpadd(oods, (q(g[0]), q(-g[1])))  # the previous row at the maximal size

    def doubled(pt, k):  # a point of the 2^L-row domain seen by a column of 2^k rows
        for _ in range(L - k):
            pt = qpadd(pt, pt)
        return pt

    sv = pr["sampled_values"]
    if [len(x) for x in sv] != [3, 4, 8, 8] or any(len(c) != 1 for tr in (0, 1, 3) for c in sv[tr]) or \
            any(len(c) != 2 for c in sv[2]):
        raise VerificationError("sampled values shape")
    pre = [qfrom(c[0]) for c in sv[0]]           # ta, tb, tc (table size)
    main = [qfrom(c[0]) for c in sv[1]]          # a, b, c (main size), m (table size)
    inter_prev = [qfrom(c[0]) for c in sv[2]]    # S_M (main size), S_T (table size)
    inter_cur = [qfrom(c[1]) for c in sv[2]]
    comp = [qfrom(c[0]) for c in sv[3]]
    basis = [q(1), q(0, 1), q(0, 0, 1), q(0, 0, 0, 1)]

    def secure(vals):
        r = q(0)
        for k in range(4):
            r = qadd(r, qmul(vals[k], basis[k]))
        return r
    left, right = secure(comp[:4]), secure(comp[4:])
    pt = oods
    for _ in range(L + 1 - 2):
        pt = qpadd(pt, pt)
    comp_eval = qadd(left, qmul(pt[0], right))
    sm, sm_prev = secure(inter_cur[:4]), secure(inter_prev[:4])
    st, st_prev = secure(inter_cur[4:]), secure(inter_prev[4:])
    d_main = qsub(qadd(qadd(main[0], qmul(alpha, main[1])), qmul(alpha2, main[2])), z)
    d_table = qsub(qadd(qadd(pre[0], qmul(alpha, pre[1])), qmul(alpha2, pre[2])), z)
    c_main = qsub(qmul(qadd(qsub(sm, sm_prev), qmulm(claimed[0], pow(1 << n, P - 2, P))), d_main), q(1))
    c_table = qadd(qmul(qadd(qsub(st, st_prev), qmulm(claimed[1], pow(1 << t, P - 2, P))), d_table), main[3])
    z_main = coset_vanishing_q(n, subgroup_gen(n + 1), subgroup_gen(n), doubled(oods, n))
    z_table = coset_vanishing_q(t, subgroup_gen(t + 1), subgroup_gen(t), doubled(oods, t))
    if qadd(qmul(qmul(random_coeff, c_main), qinv(z_main)), qmul(c_table, qinv(z_table))) != comp_eval:
        raise VerificationError("OODS mismatch")

    flat = pre + main
    for c in range(8):
        flat += [inter_prev[c], inter_cur[c]]
    flat += comp
    ch.mix_felts(flat)
    quot_coeff = ch.draw_secure_felt()
    # samples with random powers over (tree, column, sample); a two-sample column's periodicity
    # sample first, at its current point plus the lifting generator (order 2^(L+B)) doubled to the
    # column's log size (the identity for a full-size column); batches by point in order of first
    # appearance (src/core/pcs/quotients/samples.zig:163-300)
    rp = [q(1)]

    def nxt():
        r = rp[0]
        rp[0] = qmul(r, quot_coeff)
        return r
    batches = []

    def add(point, entry):
        for bp, entries in batches:
            if bp == point:
                entries.append(entry)
                return
        batches.append((point, [entry]))
    logs = [[t + B] * 3, [n + B] * 3 + [t + B], [n + B] * 4 + [t + B] * 4, [L + B] * 8]
    for c in range(3):
        add(oods, (c, pre[c], nxt()))
    for c in range(4):
        add(oods, (3 + c, main[c], nxt()))
    for c in range(8):
        k = n if c < 4 else t
        per = oods
        if k < L:
            h = index_point(1 << (31 - L + k))
            per = qpadd(oods, (q(h[0]), q(h[1])))
        add(per, (7 + c, inter_cur[c], nxt()))
        add(prev, (7 + c, inter_prev[c], nxt()))
        add(oods, (7 + c, inter_cur[c], nxt()))
    for c in range(8):
        add(oods, (15 + c, comp[c], nxt()))
    return _verify_pcs_tail(pr, ch, roots, [3, 4, 8, 8], batches, L + B, B, pow_bits, log_last, n_queries,
                            tree_logs=logs)
