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
