"""Test helpers: run the oracle for a parameter set and compare with the solver's state."""
import numpy as np

LN2_INV = 1.44269504089


def oracle_after(oracle, F, D, *, T, R, spe, beta_max, beta_ratio, seed, cap, megaiters, active=0,
                 rule=0, goal=0):
    """Oracle state after `megaiters` mega-iterations followed by each group's tracking /
    exchange step of the next mega-iteration (the solver runs that step at the end of every
    epoch, on the device, before the next launch).  active > 0: clique-flow moves; rule = 1:
    one-shot steps."""
    st = oracle.setup(D, F, T, R, spe, beta_max * LN2_INV, beta_ratio, seed, cap=cap, active=active,
                      rule=rule)
    oracle.run(st, D, F, megaiters, goal)
    oracle.track_exchange_all(st)
    return st


def compare_solver_to_oracle(solver, st, cap):
    """Returns a list of mismatch descriptions (empty when identical)."""
    bad = []
    for t in range(st.T):
        g = solver.group(t, cap)
        if not np.array_equal(g["order"], st.order[t]):
            bad.append(f"group {t} order {g['order'][:st.R]} vs {st.order[t][:st.R]}")
        if g["time_since_swap"] != st.time_since_swap[t]:
            bad.append(f"group {t} timeSinceSwap {g['time_since_swap']} vs {st.time_since_swap[t]}")
        if g["group_best"] != st.thread_best[t]:
            bad.append(f"group {t} best {g['group_best']} vs {st.thread_best[t]}")
        for l in range(st.R):
            r = solver.replica(t, l)
            for key, ref in (("E", st.E[t, l]), ("bestE", st.bestE[t, l]), ("beta", st.beta[t, l])):
                if r[key] != ref:
                    bad.append(f"replica {t}/{l} {key} {r[key]} vs {ref}")
            if not np.array_equal(r["phi"], st.phi[t, l]):
                bad.append(f"replica {t}/{l} phi differs")
            if not np.array_equal(r["I"], st.I[t, l]):
                bad.append(f"replica {t}/{l} force matrix differs")
    return bad


MASK64 = (1 << 64) - 1


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return x ^ (x >> 31)


def oracle_auto_beta(oracle, F, D, *, T, R, spe, seed, cap, lower=0.1, higher=0.9):
    """autoSelectParameters (CPU_PIM.cpp:366-476) restated on the oracle, with the solver's
    trial seeding: trial (k, t) uses splitmix64(seed + 5k + t + 1)."""
    steps, trials = 32, 5
    sums = [0.0] * steps
    denom = float(trials) * T * R
    best = None
    for i in range(steps):
        for t in range(trials):
            st = oracle.setup(D, F, T, R, spe, 2.0 ** (-30 + i), 1.0,
                              splitmix64((seed + i * trials + t + 1) & MASK64), cap=cap)
            oracle.run(st, D, F, 10)
            oracle.track_exchange_all(st)
            for g in range(T):
                for l in range(R):
                    sums[i] += float(st.E[g, l]) / denom
            b = min(int(st.bestE.min()), st.single_best)
            best = b if best is None else min(best, b)
    i = steps - 1
    minE, maxE, minEIndex = 1e30, -1e30, 0
    for j in range(i):
        if sums[j] < minE:
            minE, minEIndex = sums[j], j
        if j == 0:
            maxE = sums[j]
    minBeta = 0.0
    for j in range(i):
        if minBeta == 0 and ((j == minEIndex - 1 and j >= 1) or sums[j] < (maxE - minE) * higher + minE):
            minBeta = 2.0 ** (-30 + j)
        if j == i - 1 or (minBeta != 0 and (j == minEIndex or sums[j] < (maxE - minE) * lower + minE)):
            if minBeta == 0:
                minBeta = 2.0 ** -30
            maxBeta = 2.0 ** (-30 + j + 2)
            return maxBeta, (maxBeta / minBeta) ** (1.0 / R), sums, best
    raise AssertionError("no range")


NO_BEST = 2147483647


def oracle_cli_trace(oracle, F, D, *, T, R, spe, beta0, ratio, seed, megaiters, goal=0,
                     single=NO_BEST, cap=10):
    """What the reference's threadToRun loop (CPU_PIM.cpp:292-362) prints, restated on the
    oracle with lock-step groups: the "Best Energy Found" energies in (mega-iteration, group,
    replica) order, each group's sweep<t>.txt pairs [m, threadBestE], and the final single
    best.  `single` is the best carried in (automatic mode's trials share it)."""
    st = oracle.setup(D, F, T, R, spe, beta0, ratio, seed, cap=cap)
    thread = [NO_BEST] * T
    lines, sweeps = [], {t: [] for t in range(T)}
    for m in range(megaiters):
        bestE = st.bestE.copy()
        for t in range(T):
            found = False
            for l in range(R):
                if bestE[t, l] < thread[t]:
                    thread[t] = int(bestE[t, l])
                    found = True
                    if thread[t] < single:
                        single = thread[t]
                        lines.append(single)
            if found:
                sweeps[t].append([m, thread[t]])
        if single <= goal:
            break
        oracle.run(st, D, F, 1, -(1 << 62))
    return lines, sweeps, single
