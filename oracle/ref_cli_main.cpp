/*
 * ref_cli_main.cpp - main() of oracle/_ref/cpu_pim_philox: the reference's own CLI
 * (CPU_PIM.cpp:478-685, through ref_cli in ref_harness.cpp) with its random engine replaced by
 * the solver's Philox streams.  TEST INFRASTRUCTURE ONLY: tests/golden/make_cli_golden.py
 * runs it to record the reference's log.txt / sweep<t>.txt / stdout for the CLI parity test.
 *
 * Usage: cpu_pim_philox --seed S [the reference's flags] FILE
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" int ref_cli(uint64_t seed, int argc, char **argv);

int main(int argc, char **argv) {
    uint64_t seed = 1;
    std::vector<char *> args;
    for (int i = 0; i < argc; ++i) {
        if (i > 0 && std::strcmp(argv[i], "--seed") == 0 && i + 1 < argc) {
            seed = std::strtoull(argv[++i], nullptr, 0);
            continue;
        }
        args.push_back(argv[i]);
    }
    args.push_back(nullptr);
    return ref_cli(seed, (int)args.size() - 1, args.data());
}
