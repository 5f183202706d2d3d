"""Pure-Python oracle for small cases.  TEST INFRASTRUCTURE ONLY.

A second, independent restatement of the reference's word scan, two-hit rule
and X-drop extenders (gpu_blastp_kernel.cu:131-320 and :341-549), written for
readability rather than speed.  It keeps the diagonal state in a dict keyed by
the masked diagonal with an explicit "no hit yet" value instead of the
reference's running diagonal offset, so agreement with oracle.c also checks
that the offset trick is equivalent to a fresh table per subject.

Parity status: pinned through oracle.c, which tests/test_oracle.py checks
against this file and tests/test_ref_pinned.py against the reference's own
kernel source host-compiled into oracle/_ref (ref_driver.cpp); also pinned by
the fixture BLOSUM62 and the hand-computed cases in tests/.
"""

WORD = 3
NCELL = 1 << 15


def code3(a, b, c):
    return (int(a) << 10) | (int(b) << 5) | int(c)


def build_table(query, matrix, threshold):
    """dict code -> ascending list of query offsets (NCBI neighbour rule)."""
    cells = {}
    for q in range(len(query) - WORD + 1):
        a, b, c = query[q], query[q + 1], query[q + 2]
        self_score = matrix[a][a] + matrix[b][b] + matrix[c][c]
        for r0 in range(1, 28):
            s0 = matrix[a][r0]
            for r1 in range(1, 28):
                s1 = s0 + matrix[b][r1]
                for r2 in range(1, 28):
                    s2 = s1 + matrix[c][r2]
                    if s2 >= threshold or (self_score < threshold and (r0, r1, r2) == (a, b, c)):
                        cells.setdefault(code3(r0, r1, r2), []).append(q)
    return cells


def extend_left(matrix, subj, query, s_off, q_off, xdrop):
    """gpu_blastp_kernel.cu:435-481: returns (best score, length)."""
    n = min(s_off, q_off)
    best, best_i, score = 0, n + 1, 0
    for i in range(n, -1, -1):
        score += matrix[query[q_off - n + i]][subj[s_off - n + i]]
        if score > best:
            best, best_i = score, i
        if best - score >= xdrop:
            break
    return best, n - best_i + 1


def extend_right(matrix, subj, query, s_off, q_off, xdrop, start_score):
    """gpu_blastp_kernel.cu:503-549: returns (best score, length, s_last_off)."""
    n = min(len(subj) - s_off, len(query) - q_off)
    best, best_i, score = start_score, -1, start_score
    i = 0
    while i < n:
        score += matrix[query[q_off + i]][subj[s_off + i]]
        if score > best:
            best, best_i = score, i
        if score <= 0 or best - score >= xdrop:
            break
        i += 1
    return best, best_i + 1, s_off + i


def extend_two_hit(matrix, subj, query, s_left, s_right, q_right, xdrop):
    """gpu_blastp_kernel.cu:341-415: (hsp_q, hsp_s, len, score, s_last, right_ext)."""
    score, left_score, shift = 0, 0, 0
    for i in range(WORD):
        score += matrix[subj[s_right + i]][query[q_right + i]]
        if score > left_score:
            left_score, shift = score, i + 1
    q_right += shift
    s_right += shift
    left_score, left_d = extend_left(matrix, subj, query, s_right - 1, q_right - 1, xdrop)
    right_ext, right_d, right_score, s_last = False, 0, 0, s_right
    if left_d >= s_right - s_left:
        right_ext = True
        right_score, right_d, s_last = extend_right(matrix, subj, query, s_right, q_right,
                                                    xdrop, left_score)
    return (q_right - left_d, s_right - left_d, left_d + right_d,
            max(left_score, right_score), s_last, right_ext)


def scan_subject(subj, query, cells, matrix, contexts, window, diag_mask):
    """One subject.  contexts: list of (query_offset, xdrop, cutoff).
    Returns ((hits, successful, extended), [hsp tuples in discovery order])."""
    state = {}          # masked diagonal -> ("hit", s) or ("ext", s_last - (W-1))
    hits = ext = 0
    hsps = []
    for s in range(len(subj) - WORD + 1):
        for q in cells.get(code3(subj[s], subj[s + 1], subj[s + 2]), ()):
            hits += 1
            d = (q - s) & diag_mask
            kind, pos = state.get(d, ("none", 0))
            if kind == "ext":
                if s < pos:
                    continue
                state[d] = ("hit", s)
                continue
            if kind == "none" or s - pos >= window:
                state[d] = ("hit", s)
                continue
            if s - pos < WORD:
                continue
            k = max(i for i, c in enumerate(contexts) if c[0] <= q or i == 0)
            _, xdrop, cutoff = contexts[k]
            hq, hs, ln, sc, s_last, rext = extend_two_hit(matrix, subj, query, pos + WORD, s, q, xdrop)
            ext += 1
            if sc >= cutoff:
                hsps.append((hq, hs, q, s, ln, sc))
            state[d] = ("ext", s_last - (WORD - 1)) if rext else ("hit", s)
    return (hits, len(hsps), ext), hsps


# ---- gapped stage (conventions of oracle/gapped.h), for small cases -------

GNEG = -(1 << 28)
GWINDOW = 11


def gapped_extend(M, A, B, xdrop, go, ge):
    """One extension over A, B (walk order), rows kept as dicts of live cells."""
    best, bi, bj = 0, 0, 0
    row, frow = {0: 0}, {0: GNEG}
    e, hl = GNEG, 0
    for j in range(1, len(B) + 1):
        e = max(max(hl - go, e) - ge, GNEG)
        if e < -xdrop:
            break
        row[j], frow[j], hl = e, GNEG, e
    prev_h, prev_f = row, frow
    for i in range(1, len(A) + 1):
        lo, last = min(prev_h), max(prev_h)
        floor_prev = best - xdrop
        cur_h, cur_f = {}, {}
        e, hl = GNEG, GNEG
        j = lo
        while j <= len(B):
            up_h, up_f = prev_h.get(j, GNEG), prev_f.get(j, GNEG)
            f = max(max(up_h - go, up_f) - ge, GNEG)
            e = max(max(hl - go, e) - ge, GNEG)
            dg = prev_h.get(j - 1, GNEG)
            d = GNEG if dg == GNEG else dg + M[A[i - 1]][B[j - 1]]
            if j > last + 1 and e < floor_prev:
                break
            h = max(d, e, f)
            cur_h[j], cur_f[j], hl = h, f, h
            j += 1
        rmax = max(cur_h.values())
        rj = min(k for k, v in cur_h.items() if v == rmax)
        if rmax > best:
            best, bi, bj = rmax, i, rj
        fl = best - xdrop
        prev_h = {k: v for k, v in cur_h.items() if v >= fl}
        prev_f = {k: cur_f[k] for k in prev_h}
        if not prev_h:
            break
    return best, bi, bj


def gapped_seed(M, q, s, hq, hs, ln):
    if ln <= GWINDOW:
        return hq + ln // 2, hs + ln // 2
    wins = [sum(M[q[hq + k + t]][s[hs + k + t]] for t in range(GWINDOW)) for k in range(ln - GWINDOW + 1)]
    k = wins.index(max(wins))
    return hq + k + GWINDOW // 2, hs + k + GWINDOW // 2


def gapped_subject(M, q, s, hsps, go=11, ge=1, xdrop=38, cutoff=0):
    """hsps: the subject's ungapped HSPs (hsp_q, hsp_s, q_off, s_off, len,
    score) in discovery order.  Returns the gapped HSPs as tuples
    (score, q_start, q_end, s_start, s_end, q_seed, s_seed, ungapped)."""
    order = sorted(range(len(hsps)), key=lambda k: -hsps[k][5])   # stable: discovery order among equals
    out = []
    for k in order:
        hq, hs, _, _, ln, _ = hsps[k]
        if any(g[1] <= hq and hq + ln <= g[2] and g[3] <= hs and hs + ln <= g[4] for g in out):
            continue
        qs, ss = gapped_seed(M, q, s, hq, hs, ln)
        L, li, lj = gapped_extend(M, q[qs::-1], s[ss::-1], xdrop, go, ge)
        R, ri, rj = gapped_extend(M, q[qs + 1:], s[ss + 1:], xdrop, go, ge)
        if L + R >= cutoff:
            out.append((L + R, qs + 1 - li, qs + 1 + ri, ss + 1 - lj, ss + 1 + rj, qs, ss, k))
    return out
