// pimqap_cli.cpp - the `pimqap` command: a drop-in for the reference's CPU_PIM binary
// (CPU-PIM/CPU_PIM.cpp:478-685) on top of the C ABI only.
//
// Same flags with the same meaning (-b -g -G -h -i -m -o -r -s -t -w -al -ah), the same output
// folder (<file>.out unless -o), the same log.txt and sweep<t>.txt files and the same stdout
// lines, so the reference's drivers (CPU-PIM/run_all.py, run_timed.py) can call it unchanged.
// Added flags: --seed S (Philox key), --json PATH (best cost, permutation, time to target),
// --device D, --force-bits 32|64, --active-facilities A (the tai256c program's moves),
// --one-shot (GPU-CUPIM's one-shot parallel step instead of sequential sweeps).
//
// The solver records every group-best lowering and goal-print hit on the device with its time
// (pimqap_solver_events); this program prints them in the reference's order after each chunk
// of mega-iterations.  The reference's threads race on the shared best energy, so with more
// than one group its "Best Energy Found" lines come in a scheduling-dependent order; here they
// come in (mega-iteration, group, replica) order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "pimqap.h"

using std::cout;
using std::endl;

namespace {

using Clock = std::chrono::high_resolution_clock;

struct Options {
    int numitera = 4;                    // -i  (CPU_PIM.cpp:19)
    long long megaiters = 2147483647;    // -w  (:21)
    int replicas = 10;                   // -r  (:24)
    int threads = 20;                    // -t  (:27)
    double beta0 = std::exp2(-12);       // -b  (:29), internal units after * 1/ln2
    double delta_beta = 1.2;             // -m  (:31)
    double lower = 0.1, higher = 0.9;    // -al / -ah (:33-34)
    bool automatic = true;               // no -b (:36)
    long long goal = 0, goal_print = 0;  // -g / -G (:48-49)
    long long timeout = 0;               // -s (:50)
    std::string input, output;           // FILE / -o (:40-41)
    unsigned long long seed = 1;
    std::string json;
    int device = 0, force_bits = 0;
    int active = 0;                      // --active-facilities: the tai256c program's moves
    bool one_shot = false;               // --one-shot: GPU-CUPIM's parallel step
};

void usage(const char *argv0) {   // :486-503
    cout << "Usage: " << argv0 << " [OPTIONS]... [FILE]..." << endl;
    cout << "Tries to find solution to provided Quadratic Assignment Problem (QAP) file" << endl;
    cout << endl;
    cout << "-b              set the beta of the largest beta replica" << endl;
    cout << "-g              set the goal objective value, program halts when reached" << endl;
    cout << "-G              set the goal objective value, prints solution when reached" << endl;
    cout << "-h, --help      displays this help message and exits" << endl;
    cout << "-i              set number of iterations between replica swaps, defaults to 4" << endl;
    cout << "-m              set the multiplative difference in beta replicas" << endl;
    cout << "-o              set the output folder name" << endl;
    cout << "-r              set number of repulicas, defaults to maximum compiled for" << endl;
    cout << "-s              set the timeout in seconds, program halts when reached" << endl;
    cout << "-t              set number of threads, defaults to maximum compiled for" << endl;
    cout << "-w              set number of swaps, program halts when reached" << endl;
    cout << endl;
    cout << "If -b is not set, then automatic mode is used." << endl;
    cout << "In automatic mode, a series of short trials at different betas are used to try and choose the best parameters." << endl;
    cout << endl;
    cout << "Additional options:" << endl;
    cout << "--seed S        key of the counter-based random stream (default 1)" << endl;
    cout << "--json PATH     write the best cost, permutation and time to target as JSON" << endl;
    cout << "--device D      CUDA device ordinal (default 0)" << endl;
    cout << "--force-bits B  force-matrix width 32 or 64 (default: from the instance bound)" << endl;
    cout << "--active-facilities A  the moves of the reference's CPU_PIM_tai256c program: facilities" << endl;
    cout << "                0..A-1 form a clique of unit flows, the others carry none (A = 92 there)" << endl;
    cout << "--one-shot      GPU-CUPIM's one-shot step: every location proposes at once, collisions" << endl;
    cout << "                go to the larger delta (a sweep is one such step; needs -b)" << endl;
}

// std::stoi / std::stod as the reference uses them, with a message instead of an abort.
bool to_ll(const std::string &flag, const char *s, long long *out) {
    try {
        *out = std::stoll(s);
        return true;
    } catch (...) {
        std::cerr << "Error: " << flag << " option requires a numeric value." << endl;
        return false;
    }
}

bool to_d(const std::string &flag, const char *s, double *out) {
    try {
        *out = std::stod(s);
        return true;
    } catch (...) {
        std::cerr << "Error: " << flag << " option requires a numeric value." << endl;
        return false;
    }
}

// Parses argv like CPU_PIM.cpp:481-606.  Returns -1 to go on, else the exit code.  Unlike the
// reference, -al / -ah are not also taken as the file name (:507-525 fall through to :604).
int parse(int argc, char **argv, Options &o) {
    for (int i = 1; i < argc; ++i) {
        const std::string arg = argv[i];
        auto value = [&]() -> const char * {
            if (i + 1 < argc) return argv[++i];
            std::cerr << "Error: " << arg << " option requires a value." << endl;
            return nullptr;
        };
        const char *s = nullptr;
        long long v = 0;
        double d = 0;
        if (arg == "--help" || arg == "-h") {
            usage(argv[0]);
            return 0;
        } else if (arg == "-al") {
            if (!(s = value()) || !to_d(arg, s, &o.lower)) return 1;
        } else if (arg == "-ah") {
            if (!(s = value()) || !to_d(arg, s, &o.higher)) return 1;
        } else if (arg == "-b") {
            if (!(s = value()) || !to_d(arg, s, &d)) return 1;
            o.beta0 = d * 1.44269504089;   // :528
            o.automatic = false;
        } else if (arg == "-g") {
            if (!(s = value()) || !to_ll(arg, s, &o.goal)) return 1;
        } else if (arg == "-G") {
            if (!(s = value()) || !to_ll(arg, s, &o.goal_print)) return 1;
        } else if (arg == "-i") {
            if (!(s = value()) || !to_ll(arg, s, &v)) return 1;
            o.numitera = (int)v;
        } else if (arg == "-m") {
            if (!(s = value()) || !to_d(arg, s, &o.delta_beta)) return 1;
        } else if (arg == "-o") {
            if (!(s = value())) return 1;
            o.output = s;
        } else if (arg == "-r") {
            if (!(s = value()) || !to_ll(arg, s, &v)) return 1;
            o.replicas = (int)v;
            if (o.replicas > PIMQAP_MAX_REPLICAS) {   // :572-576
                std::cerr << "Error: -r option exceeds maximum number of replicas (" << PIMQAP_MAX_REPLICAS << ")." << endl;
                return 1;
            }
        } else if (arg == "-s") {
            if (!(s = value()) || !to_ll(arg, s, &o.timeout)) return 1;
        } else if (arg == "-t") {
            if (!(s = value()) || !to_ll(arg, s, &v)) return 1;
            o.threads = (int)v;
            if (o.threads > PIMQAP_MAX_GROUPS) {      // :591-595
                std::cerr << "Error: -t option exceeds maximum number of threads (" << PIMQAP_MAX_GROUPS << ")." << endl;
                return 1;
            }
        } else if (arg == "-w") {
            if (!(s = value()) || !to_ll(arg, s, &o.megaiters)) return 1;
        } else if (arg == "--seed") {
            if (!(s = value())) return 1;
            try {
                o.seed = std::stoull(s, nullptr, 0);
            } catch (...) {
                std::cerr << "Error: --seed option requires a numeric value." << endl;
                return 1;
            }
        } else if (arg == "--json") {
            if (!(s = value())) return 1;
            o.json = s;
        } else if (arg == "--device") {
            if (!(s = value()) || !to_ll(arg, s, &v)) return 1;
            o.device = (int)v;
        } else if (arg == "--active-facilities") {
            if (!(s = value()) || !to_ll(arg, s, &v)) return 1;
            o.active = (int)v;
        } else if (arg == "--one-shot") {
            o.one_shot = true;
        } else if (arg == "--force-bits") {
            if (!(s = value()) || !to_ll(arg, s, &v)) return 1;
            o.force_bits = (int)v;
        } else {
            o.input = arg;   // the last positional argument is the file (:604)
        }
    }
    return -1;
}

long long ms_since(Clock::time_point t0) {
    return std::chrono::duration_cast<std::chrono::milliseconds>(Clock::now() - t0).count();
}

// The reference's tracking state (threadBestE, singleBestE) and the lines it prints from it.
struct Tracker {
    std::ofstream &log;
    std::vector<std::ofstream> *sweep = nullptr;   // sweep<t>.txt (null during automatic mode)
    std::vector<long long> thread_best;
    long long single_best = 2147483647;           // :55, carried over from automatic mode
    double offset_ms = 0;                         // host ms from startTime to the event clock's zero
    long long goal = 0;
    double target_ms = -1;                        // when single_best first reached the goal

    Tracker(std::ofstream &l, int groups, long long g) : log(l), thread_best(groups, 2147483647LL), goal(g) {}

    // Group-best events of one solve, in (mega-iteration, group, replica) order; events at or
    // after `limit` were seen by a tracking step the reference never runs and are skipped.
    void group_best(const pimqap_event *ev, int count, long long limit) {
        for (int k = 0; k < count; ++k) {
            const pimqap_event &e = ev[k];
            if (e.kind != PIMQAP_EVENT_GROUP_BEST || e.megaiter >= limit) continue;
            thread_best[e.group] = e.energy;                              // :298-301
            const long long ms = (long long)(offset_ms + e.time_ms);
            if (e.energy < single_best) {                                 // :303-311
                single_best = e.energy;
                if (single_best <= goal && target_ms < 0) target_ms = offset_ms + e.time_ms;
                log << "Best Energy Found: " << single_best << " Time (s): " << ms / 1000.0 << endl;
                cout << "Best Energy Found: " << single_best << " Time (s): " << ms / 1000.0 << endl;
            }
            const bool last_of_group = k + 1 == count || ev[k + 1].kind != PIMQAP_EVENT_GROUP_BEST ||
                                       ev[k + 1].megaiter != e.megaiter || ev[k + 1].group != e.group ||
                                       ev[k + 1].trial != e.trial;
            if (last_of_group && sweep)                                   // :316-321
                (*sweep)[e.group] << e.megaiter << " " << ms << " " << thread_best[e.group] << endl;
        }
    }
};

int fail_api(const char *what) {
    std::cerr << "Error: " << what << ": " << pimqap_last_error() << endl;
    return 1;
}

int run(int argc, char **argv) {
    Options o;
    const int rc = parse(argc, argv, o);
    if (rc >= 0) return rc;
    if (o.input.empty()) {                                           // :608-611
        std::cerr << "Error: No input file specified." << endl;
        return 1;
    }
    if (o.output.empty()) o.output = o.input + ".out";               // :613-615
    try {                                                            // :617-631
        if (!std::filesystem::create_directory(o.output))
            std::cerr << "Error: Folder '" << o.output << "' already exists or could not be created." << std::endl;
    } catch (const std::filesystem::filesystem_error &e) {
        std::cerr << "Error: Error creating folder: " << e.what() << std::endl;
        return 1;
    }
    {                                                                // readProblem (:79-107)
        std::ifstream probe(o.input);
        if (!probe.is_open()) {
            std::cerr << "Error: Could not open the file (" << o.input << ")." << endl;
            return 1;
        }
    }
    int32_t n = 0;
    pimqap_status st = pimqap_read_problem(o.input.c_str(), PIMQAP_MAX_N, &n, nullptr, nullptr);
    if (st == PIMQAP_ERR_ARG) {
        std::cerr << "Error: N exceeded MAXN (" << PIMQAP_MAX_N << ")." << endl;
        return 1;
    }
    std::vector<int32_t> flow, dist;
    if (st == PIMQAP_OK) {
        flow.resize((size_t)n * n);
        dist.resize((size_t)n * n);
        st = pimqap_read_problem(o.input.c_str(), PIMQAP_MAX_N, &n, flow.data(), dist.data());
    }
    if (st != PIMQAP_OK) return fail_api("reading the instance");
    const pimqap_instance inst{n, flow.data(), dist.data()};

    pimqap_params p;
    pimqap_default_params(&p);
    p.replicas = o.replicas;
    p.groups = o.threads;
    p.sweeps_per_exchange = o.numitera;
    p.goal = o.goal;
    p.seed = o.seed;
    p.device = o.device;
    p.force_bits = o.force_bits;
    p.active_facilities = o.active;
    p.update_rule = o.one_shot ? PIMQAP_RULE_ONE_SHOT : PIMQAP_RULE_SEQUENTIAL;
    p.auto_lower = o.lower;
    p.auto_higher = o.higher;
    p.beta_internal = 1;
    p.beta_max = o.beta0;
    p.beta_ratio = o.delta_beta;
    p.goal_print = o.goal_print;
    p.event_capacity = 1 << 20;
    p.max_megaiters = o.megaiters;

    const auto start = Clock::now();                                 // :638
    std::ofstream log(o.output + "/log.txt");                        // :640-644
    log << "Iterations between swaps " << o.numitera << endl
        << "Number of Swaps " << o.megaiters << endl
        << "Number of Replicas " << o.replicas << endl
        << "Number of Threads " << o.threads << endl;
    Tracker tr(log, o.threads, o.goal);
    double beta0 = o.beta0, delta_beta = o.delta_beta;
    long long auto_best = PIMQAP_NO_BEST;
    std::vector<int32_t> auto_perm(n);
    if (!o.automatic) {                                              // :645-649
        log << "Maximum Beta " << beta0 << endl << "Multiplicative Beta between iterations " << delta_beta << endl;
        cout << "Maximum Beta " << beta0 << endl << "Multiplicative Beta between iterations " << delta_beta << endl;
    } else {                                                         // :650-658, :373-476
        log << "Automatic mode enabled, Beta parameters will be determined automatically." << endl;
        std::vector<pimqap_event> ev(1 << 20);
        pimqap_auto_report rep;
        std::memset(&rep, 0, sizeof(rep));
        rep.best_perm = auto_perm.data();
        rep.events = ev.data();
        rep.event_capacity = (int32_t)ev.size();
        const double t_auto = (double)ms_since(start);
        st = pimqap_auto_beta_report(&inst, &p, &rep);
        if (st != PIMQAP_OK) return fail_api("automatic mode");
        if (rep.events_dropped) std::cerr << "Warning: " << rep.events_dropped << " automatic-mode events not shown." << endl;
        tr.offset_ms = t_auto;
        // the trials ran in one launch; their lines are printed in the reference's trial order
        int k = 0;
        const int used_trials = rep.goal_trial >= 0 ? rep.goal_trial + 1 : PIMQAP_AUTO_STEPS * PIMQAP_AUTO_TRIALS;
        for (int trial = 0; trial < used_trials; ++trial) {
            const int first = k;
            while (k < rep.event_count && rep.events[k].trial == trial) ++k;
            std::fill(tr.thread_best.begin(), tr.thread_best.end(), 2147483647LL);   // setup() (:129)
            tr.group_best(rep.events + first, k - first, 10);
            const int step = trial / PIMQAP_AUTO_TRIALS;
            if (trial % PIMQAP_AUTO_TRIALS == PIMQAP_AUTO_TRIALS - 1 && step < rep.steps_printed) {
                log << "Beta: " << std::exp2(-30.0 + step) << ", Average Energy: " << rep.avg_energy[step] << endl;
                cout << "Beta: " << std::exp2(-30.0 + step) << ", Average Energy: " << rep.avg_energy[step] << endl;
            }
        }
        auto_best = rep.best_energy;
        if (rep.goal_trial < 0) {
            if (rep.min_beta_printed) {
                log << "Selecting minimum beta of " << rep.min_beta << endl;
                cout << "Selecting minimum beta of " << rep.min_beta << endl;
            }
            log << "Selecting maximum beta of " << rep.max_beta << endl;
            cout << "Selecting maximum beta of " << rep.max_beta << endl;
            const long long secs = ms_since(start) / 1000;
            log << "Selecting Beta Parameters took " << secs << " seconds." << endl;
            cout << "Selecting Beta Parameters took " << secs << " seconds." << endl << endl;
        }
        beta0 = rep.beta0_internal;
        delta_beta = rep.delta_beta;
        log << "Maximum Beta " << beta0 << endl << "Multiplicative Beta between iterations " << delta_beta << endl;
        cout << "Maximum Beta " << beta0 << endl << "Multiplicative Beta between iterations " << delta_beta << endl;
    }
    log << "Input file: " << o.input << endl;                        // :659

    pimqap_result res;
    std::memset(&res, 0, sizeof(res));
    std::vector<int32_t> best_perm(n);
    res.best_perm = best_perm.data();
    long long megaiters_done = 0;
    bool ran = false;
    if (!(tr.single_best <= o.goal)) {                               // :661-674
        std::vector<std::ofstream> sweep(o.threads);
        for (int t = 0; t < o.threads; ++t) sweep[t].open(o.output + "/sweep" + std::to_string(t) + ".txt");
        tr.sweep = &sweep;
        std::fill(tr.thread_best.begin(), tr.thread_best.end(), 2147483647LL);
        p.beta_max = beta0;
        p.beta_ratio = delta_beta;
        p.auto_beta = 0;
        pimqap_solver *s = nullptr;
        st = pimqap_solver_create(&inst, &p, &s);
        if (st != PIMQAP_OK) return fail_api("solver set-up");
        tr.offset_ms = (double)ms_since(start);
        ran = true;
        const int chunk = 50;
        std::vector<pimqap_event> ev;
        int64_t seen = 0, reported_drops = 0;
        long long left = o.megaiters;
        bool stop = false;
        while (!stop) {
            if (left > 0) {
                st = pimqap_solver_run(s, std::min<long long>(left, chunk), nullptr);
                if (st != PIMQAP_OK) break;
            }
            pimqap_result r;
            std::memset(&r, 0, sizeof(r));
            st = pimqap_solver_result(s, &r);
            if (st != PIMQAP_OK) break;
            left = o.megaiters - r.megaiters_done;
            {   // print what the chunk recorded (all of it: a (mega-iteration, group) run of events
                // is never split)
                int32_t cnt = 0;
                int64_t total = 0, dropped = 0;
                st = pimqap_solver_events(s, 0, 0, nullptr, &cnt, &total, &dropped);
                if (st != PIMQAP_OK) break;
                ev.resize((size_t)std::max<int64_t>(1, total - seen));
                st = pimqap_solver_events(s, seen, (int32_t)(total - seen), ev.data(), &cnt, nullptr, nullptr);
                if (st != PIMQAP_OK) break;
                for (int k = 0; k < cnt; ++k) {
                    const pimqap_event &e = ev[k];
                    if (e.kind == PIMQAP_EVENT_GROUP_BEST) {
                        int j = k;
                        while (j + 1 < cnt && ev[j + 1].kind == PIMQAP_EVENT_GROUP_BEST) ++j;
                        tr.group_best(ev.data() + k, j - k + 1, o.megaiters);
                        k = j;
                    } else {                                          // :271-282
                        log << "Thread " << e.group << " Replica " << e.replica << ": Goal surpassed: " << e.energy << endl;
                        cout << "Thread " << e.group << " Replica " << e.replica << ": Goal surpassed: " << e.energy << endl;
                        std::vector<int32_t> perm(n);
                        if (e.perm_index >= 0 && pimqap_solver_event_perm(s, e.perm_index, perm.data()) == PIMQAP_OK) {
                            for (int i = 0; i < n; ++i) {
                                log << perm[i] << " ";
                                cout << perm[i] << " ";
                            }
                        }
                        log << endl;
                        cout << endl;
                    }
                }
                seen += cnt;
                if (dropped > reported_drops) {
                    std::cerr << "Warning: " << dropped - reported_drops << " progress events not shown." << endl;
                    reported_drops = dropped;
                }
            }
            megaiters_done = r.megaiters_done;
            if (r.stopped_by == 1 || left <= 0) stop = true;          // goal (:346) or -w (:293)
            if (o.timeout > 0 && ms_since(start) / 1000 >= o.timeout) stop = true;   // :350-357
        }
        if (st == PIMQAP_OK) st = pimqap_solver_result(s, &res);
        if (st != PIMQAP_OK) {
            const int code = fail_api("solve");
            pimqap_solver_destroy(s);
            return code;
        }
        pimqap_solver_destroy(s);
        for (auto &f : sweep) f.close();
    }
    const long long single = tr.single_best;
    cout << endl;                                                    // :676-684
    cout << "Halting program." << endl;
    log << "Single best energy found: " << single << endl;
    cout << "Single best energy found: " << single << endl;
    cout << "AFD " << (1.0 * single - o.goal) / o.goal * 100.0 << endl;
    const long long el = ms_since(start);
    log << "Elapsed time: " << el / 1000.0 << " seconds." << endl;
    cout << "Elapsed time: " << el / 1000.0 << " seconds." << endl;

    if (!o.json.empty()) {
        // best state seen anywhere (the last mega-iteration's sweeps included), beside the
        // reference-equivalent tracked best printed above
        long long best_any = ran ? (long long)res.best_energy : (long long)PIMQAP_NO_BEST;
        const int32_t *bp = best_perm.data();
        if (o.automatic && auto_best < best_any) {
            best_any = auto_best;
            bp = auto_perm.data();
        }
        std::ofstream js(o.json);
        js << "{\"best_energy\": " << best_any << ", \"single_best_energy\": " << single << ", \"best_perm\": [";
        if (best_any != PIMQAP_NO_BEST)
            for (int i = 0; i < n; ++i) js << (i ? ", " : "") << bp[i];
        js << "], \"goal\": " << o.goal << ", \"time_to_target_s\": ";
        if (tr.target_ms >= 0) js << tr.target_ms / 1000.0;
        else js << "null";
        js << ", \"megaiters\": " << megaiters_done << ", \"elapsed_s\": " << el / 1000.0
           << ", \"beta_max\": " << beta0 << ", \"beta_ratio\": " << delta_beta << ", \"seed\": " << o.seed << "}" << endl;
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv) { return run(argc, argv); }
