"""Test helpers: run the oracle for a parameter set and compare with the solver's state."""
import numpy as np

LN2_INV = 1.44269504089


def oracle_after(oracle, F, D, *, T, R, spe, beta_max, beta_ratio, seed, cap, megaiters):
    """Oracle state after `megaiters` mega-iterations followed by each group's tracking /
    exchange step of the next mega-iteration (the solver runs that step at the end of every
    epoch, on the device, before the next launch)."""
    st = oracle.setup(D, F, T, R, spe, beta_max * LN2_INV, beta_ratio, seed, cap=cap)
    oracle.run(st, D, F, megaiters)
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
