"""Records the reference CLI's outputs for the CLI parity test (tests/test_cli.py).

TEST INFRASTRUCTURE.  Runs oracle/_ref/cpu_pim_philox -- the reference's own CPU_PIM main()
(CPU-PIM/CPU_PIM.cpp:478-685) built from its source by oracle/build_ref.sh, with its random
engine fed the solver's Philox streams -- on small synthetic instances and writes, per case,
its stdout, log.txt and sweep<t>.txt with the wall-clock figures blanked out, into
cli_golden.json beside this script.  The instance files (cli/*.dat) are written here too, from
the package's seeded generators.

Run from the repository root after `make -C oracle`:  python tests/golden/make_cli_golden.py
"""
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "p-dit-probabilistic-ising-machine-for-solving-the-quadratic-assignment-problem_b200"))
import instances  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "cpu_pim_philox")
STOCK = os.path.join(ROOT, "oracle", "_ref", "cpu_pim_stock")

# (name, instance file, seed, flags, deterministic line order).  The reference runs one
# std::thread per group and they race on the shared best, so with -t > 1 only the sweep files
# and the final best are order-free.
CASES = [
    ("fixed_t1", "u24.dat", 9, ["-b", "0.0002", "-m", "1.3", "-r", "4", "-t", "1", "-i", "2", "-w", "60"], True),
    ("fixed_t3", "u24.dat", 9, ["-b", "0.0002", "-m", "1.3", "-r", "4", "-t", "3", "-i", "2", "-w", "60"], False),
    ("fixed_t2_i1", "h20.dat", 4, ["-b", "0.01", "-m", "1.25", "-r", "6", "-t", "2", "-i", "1", "-w", "80"], False),
    ("goal_t1", "u24.dat", 9, ["-b", "0.0002", "-m", "1.3", "-r", "4", "-t", "1", "-i", "2", "-w", "100000",
                                "-g", "@goal"], True),
    ("goalprint_t1", "u24.dat", 9, ["-b", "0.0002", "-m", "1.3", "-r", "4", "-t", "1", "-i", "2", "-w", "60",
                                     "-G", "@goal_print"], True),
    ("auto_t1", "u12.dat", 3, ["-r", "4", "-t", "1", "-i", "1", "-w", "30"], True),
    ("auto_al_ah_t1", "u12.dat", 5, ["-al", "0.0", "-ah", "0.4", "-r", "3", "-t", "1", "-i", "2", "-w", "20"], True),
    ("auto_goal_t1", "u12.dat", 3, ["-r", "4", "-t", "1", "-i", "1", "-w", "30", "-g", "@auto_goal"], True),
]

TIME = re.compile(r"(Time \(s\): )\S+")
ELAPSED = re.compile(r"^(Elapsed time: )\S+( seconds\.)$")
TOOK = re.compile(r"^(Selecting Beta Parameters took )\d+( seconds\.)$")


def normalise(text):
    out = []
    for line in text.splitlines():
        line = TIME.sub(r"\1*", line)
        line = ELAPSED.sub(r"\1*\2", line)
        line = TOOK.sub(r"\1*\2", line)
        out.append(line)
    return out


def sweep_pairs(path):
    """sweep<t>.txt lines 'm ms best' as [m, best] (the ms column is wall time)."""
    pairs = []
    with open(path) as f:
        for line in f:
            m, _ms, best = line.split()
            pairs.append([int(m), int(best)])
    return pairs


def run_ref(inst_path, seed, flags, workdir):
    out = os.path.join(workdir, "out")
    cp = subprocess.run([REF, "--seed", str(seed)] + flags + ["-o", out, inst_path],
                        capture_output=True, text=True, check=True, timeout=600)
    with open(os.path.join(out, "log.txt")) as f:
        log = f.read()
    sweeps = {}
    for name in sorted(os.listdir(out)):
        m = re.fullmatch(r"sweep(\d+)\.txt", name)
        if m:
            sweeps[m.group(1)] = sweep_pairs(os.path.join(out, name))
    return cp.stdout, log, sweeps


def best_lines(stdout):
    return [int(l.split()[3]) for l in stdout.splitlines() if l.startswith("Best Energy Found:")]


def main():
    if not os.path.exists(REF):
        sys.exit(f"{REF} is not built (make -C oracle)")
    files = {
        "u24.dat": instances.uniform(24, 77),
        "u12.dat": instances.uniform(12, 31),
        "h20.dat": instances.heavy(20, 5),
    }
    for name, inst in files.items():
        instances.write_instance(os.path.join(HERE, "cli", name), inst)
    rel = lambda name: os.path.join("tests", "golden", "cli", name)  # noqa: E731

    # placeholders resolved from runs without them
    with tempfile.TemporaryDirectory() as d:
        so, _, _ = run_ref(rel("u24.dat"), 9, CASES[0][3], d)
    lines = best_lines(so)
    resolved = {"@goal": str(lines[len(lines) // 2]), "@goal_print": str(lines[-3])}
    with tempfile.TemporaryDirectory() as d:
        so, _, _ = run_ref(rel("u12.dat"), 3, CASES[5][3], d)
    auto_lines = [l for l in so.splitlines() if l.startswith("Best Energy Found:")]
    resolved["@auto_goal"] = str(best_lines(so)[min(4, len(auto_lines) - 1)])

    cases = []
    for name, inst_file, seed, flags, ordered in CASES:
        flags = [resolved.get(f, f) for f in flags]
        with tempfile.TemporaryDirectory() as d:
            so, log, sweeps = run_ref(rel(inst_file), seed, flags, d)
        cases.append(dict(name=name, instance=inst_file, seed=seed, flags=flags, ordered=ordered,
                          stdout=normalise(so), log=normalise(log), sweeps=sweeps))
        print(f"{name}: {len(so.splitlines())} stdout lines, {len(sweeps)} sweep files")
    help_text = subprocess.run([STOCK, "--help"], capture_output=True, text=True, check=True).stdout
    doc = dict(generator="tests/golden/make_cli_golden.py", reference="CPU-PIM/CPU_PIM.cpp main()",
               help=help_text.splitlines()[1:], cases=cases)
    with open(os.path.join(HERE, "cli_golden.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
