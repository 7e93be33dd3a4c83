"""CPU restatement of RabbitBin's label propagation (test infrastructure only).

Pure-Python loops, for small graphs: tests compare it with the reference's own
code (oracle/_ref, ref_label_propagation) and with the device sweep.  It follows
  * the incidence build, src/rabbitbin.cpp:5597-5622 (edges with a score above
    0, clamped to 1 - 1e-6f, both endpoints' lists ordered by neighbour id);
  * the per-edge quantity, src/impl/rb_cluster.cpp:449-454 ((float)log(1 - w)
    or the score itself for the sum / mean / max rules);
  * the score rules and chi-squared tail, src/impl/rb_cluster.cpp:3-22, :40-76;
  * the sequential sweep, src/impl/rb_cluster.cpp:596-714, and the
    synchronous one, :490-594.
Python's math.exp and math.log are the C library's, as in the reference.
"""
import math

import numpy as np

RULES = {"fisher": 0, "tail": 1, "logsum": 2, "sum": 3, "mean": 4, "max": 5}
SSCR_MAX = float(np.float32(1.0) - np.float32(1e-6))
EPS = 1e-12


def _chi2_sf(m, x):
    u = 0.5 * x
    p = math.exp(-u)
    q = p
    for i in range(1, m):
        p *= u / float(i)
        q += p
    return q


def _combine(rule, m, acc):
    if rule == 0:
        v = 1.0 - _chi2_sf(m, -2.0 * acc)
        return 0.0 if v < 0.0 else v
    if rule == 1:
        return -_chi2_sf(m, -2.0 * acc)
    if rule == 2:
        return -acc
    if rule == 4:
        return acc / float(m) if m > 0 else 0.0
    return acc


def incidence(n, src, dst, score, rule=0):
    """Neighbour lists [(neighbour, quantity)] in the reference's order."""
    raw = rule in (3, 4, 5)
    lists = [[] for _ in range(n)]
    for e in range(len(src)):
        w = float(np.float32(score[e]))
        if not w > 0.0:
            continue
        if w > SSCR_MAX:
            w = SSCR_MAX
        q = w if raw else float(np.float32(math.log(1.0 - w)))
        a, b = int(src[e]), int(dst[e])
        lists[a].append((b, e, q))
        lists[b].append((a, e, q))
    return [[(u, q) for u, _, q in sorted(l, key=lambda t: (t[0], t[1]))] for l in lists]


def _decide(rule, arcs, label, cur):
    score, count, touched = {}, {}, []
    for u, q in arcs:
        k = label[u]
        if k not in count:
            touched.append(k)
            score[k], count[k] = 0.0, 0
        if rule == 5:
            if q > score[k]:
                score[k] = q
        else:
            score[k] += q
        count[k] += 1
    if not touched:
        return None
    best_v, best_k, cur_v = -math.inf, touched[0], None
    for k in touched:
        v = _combine(rule, count[k], score[k])
        if k == cur:
            cur_v = v
        if v > best_v:
            best_v, best_k = v, k
    if cur_v is not None and cur_v >= best_v - EPS:
        best_k = cur
    return best_k


def label_propagation(n, src, dst, score, order, rule=0, synchronous=False):
    """Labels after propagation; order is the node order (a permutation)."""
    lists = incidence(n, src, dst, score, rule)
    label = list(range(n))
    if n == 0 or len(src) == 0:
        return np.array(label, np.uint32)
    visited, frozen = {}, set()

    def change(v, kprev, best):
        label[v] = best
        seen = visited.setdefault(v, set())
        if not seen:
            seen.add(kprev)
        if best in seen:
            frozen.add(v)
        else:
            seen.add(best)

    active = [True] * n
    while True:
        changed = 0
        if synchronous:
            prop = {}
            for v in order:
                if active[v]:
                    b = _decide(rule, lists[v], label, label[v])
                    if b is not None:
                        prop[v] = b
            nxt = [False] * n
            for v in order:
                if v in prop and label[v] != prop[v] and v not in frozen:
                    for u, _ in lists[v]:
                        nxt[u] = True
                    change(v, label[v], prop[v])
                    changed += 1
            active = nxt
        else:
            for v in order:
                if not active[v]:
                    continue
                active[v] = False
                b = _decide(rule, lists[v], label, label[v])
                if b is not None and b != label[v] and v not in frozen:
                    for u, _ in lists[v]:
                        active[u] = True
                    change(v, label[v], b)
                    changed += 1
        if changed == 0:
            break
    return np.array(label, np.uint32)
