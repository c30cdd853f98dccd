// TEST INFRASTRUCTURE ONLY.  Drives GPU-CUPIM's own one-shot step (perl-gpu/src/lib/qap/qap.cu:
// ReplicaPool::perform_step_one_shot, :1462-1600, with the kernels os_pwc_d :1038-1146,
// os_resolve_{i,ii,iii}_d :1150-1225, os_update_force_mats_d :1336-1412, os_apply_swaps_ii_d
// :1310-1332 and os_score_from_force_mat_d :1419-1458) from Python through ctypes, so that the
// oracle's restatement of the one-shot rule (orc_oneshot_step, oracle/pim_oracle.c) can be pinned
// against the reference's kernels on the same states and the same uniforms.
//
// The reference source is compiled where it lies (oracle/build_cupim.sh puts its qap/ directory
// on the include path); the only substitution is its random-number header (cupim_shim/random.cuh:
// cuRANDDx is not available), whose generator copies the uniforms this harness uploads.  The
// solver library never links this.
//
// Pool: width R, depth 1, F = float, Z = int32 (qap_gpu.cu's defaults without --large-energies).
// Every entry point returns 0 on success and a negative code otherwise.
#include "qap.cu"

#include <cstdint>
#include <cstring>
#include <vector>

namespace {
using Pool = qap::ReplicaPool<float, int32_t>;
Pool g_host, g_dev;
bool g_open = false;
float4 *g_uni = nullptr;
uint32_t g_n = 0, g_R = 0;

int cuda_ok(cudaError_t e) { return e == cudaSuccess ? 0 : -100 - (int)e; }
}  // namespace

// Opens a pool of R replicas on the instance file at `path` (n, then F, then D: the reference's
// format, read by its own Layout::from_file).  n must be 1..256 (os_pwc_d's limit).
extern "C" int cupim_open(const char *path, int R) {
    if (g_open || R < 1) return -1;
    g_host = Pool::from_file(path, (uint32_t)R, 1, 1.0f, 1.0f);
    g_n = g_host.invariants.problem_size;
    g_R = (uint32_t)R;
    if (g_n < 1 || g_n > 256) {
        g_host.cu_free();
        return -2;
    }
    // from_file leaves the layout's own permutation arrays zero-length, while cu_copy copies n
    // entries of them: give them n entries first
    delete[] g_host.invariants.facility_at_position;
    delete[] g_host.invariants.position_of_facility;
    g_host.invariants.facility_at_position = new uint32_t[g_n];
    g_host.invariants.position_of_facility = new uint32_t[g_n];
    for (uint32_t i = 0; i < g_n; ++i)
        g_host.invariants.facility_at_position[i] = g_host.invariants.position_of_facility[i] = i;
    g_dev = g_host.cu_copy(cudaMemcpyHostToDevice);
    const size_t nq = ((size_t)g_R * g_n + 3) / 4;
    int rc = cuda_ok(cudaMalloc(&g_uni, nq * sizeof(float4)));
    if (!rc) rc = cuda_ok(cudaMemset(g_uni, 0, nq * sizeof(float4)));
    if (!rc) rc = cuda_ok(cudaMemcpyToSymbol(g_pin_uniforms, &g_uni, sizeof(g_uni)));
    if (!rc) rc = cuda_ok(cudaDeviceSynchronize());
    if (rc) {   // leave nothing behind: a later open starts clean
        g_dev.cu_free();
        g_host.cu_free();
        cudaFree(g_uni);
        g_uni = nullptr;
        return rc;
    }
    g_open = true;
    return 0;
}

// Sets every replica's permutation (phi[r][i] = facility at location i) and beta, then lets the
// reference recompute the force matrices and energies on the device (recompute_force_mats(32),
// recompute_energies<32>(), as qap_gpu.cu:483-484 does after loading).
extern "C" int cupim_set(const int32_t *phi, const float *betas) {
    if (!g_open) return -1;
    const uint32_t n = g_n;
    for (uint32_t r = 0; r < g_R; ++r) {
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t a = (uint32_t)phi[(size_t)r * n + i];
            if (a >= n) return -2;
            g_host.facility_at_position[r * n + i] = a;
            g_host.position_of_facility[r * n + a] = i;
        }
        g_host.betas[r] = betas[r];
        g_host.best_score_per_replica[r] = INT32_MAX;
    }
    g_host.best_score_per_deck[0] = INT32_MAX;
    g_host.best_score_overall[0] = INT32_MAX;
    const size_t rn = (size_t)g_R * n;
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    int rc = cuda_ok(cudaMemcpy(g_dev.facility_at_position, g_host.facility_at_position, rn * 4, h2d));
    if (!rc) rc = cuda_ok(cudaMemcpy(g_dev.position_of_facility, g_host.position_of_facility, rn * 4, h2d));
    if (!rc) rc = cuda_ok(cudaMemcpy(g_dev.betas, g_host.betas, g_R * sizeof(float), h2d));
    if (!rc) rc = cuda_ok(cudaMemcpy(g_dev.best_score_per_replica, g_host.best_score_per_replica, g_R * 4, h2d));
    if (!rc) rc = cuda_ok(cudaMemcpy(g_dev.best_score_per_deck, g_host.best_score_per_deck, 4, h2d));
    if (!rc) rc = cuda_ok(cudaMemcpy(g_dev.best_score_overall, g_host.best_score_overall, 4, h2d));
    if (rc) return rc;
    g_dev.recompute_force_mats(32);
    g_dev.template recompute_energies<32>();
    return cuda_ok(cudaDeviceSynchronize());
}

// One one-shot step of every replica with the uniforms u[r][i] (the threshold of location i of
// replica r), through the reference's own graph (perform_step_one_shot<1024>, the block size
// qap_gpu.cu:248 uses; the seed only feeds the replaced generator).
extern "C" int cupim_step(const float *u) {
    if (!g_open) return -1;
    int rc = cuda_ok(cudaMemcpy(g_uni, u, sizeof(float) * (size_t)g_R * g_n, cudaMemcpyHostToDevice));
    if (rc) return rc;
    g_dev.template perform_step_one_shot<1024>(0);
    return cuda_ok(cudaDeviceSynchronize());
}

// Reads back the permutations, force matrices ([r][i][a]), energies (replica_score) and the
// step's resolved proposals (proposed_targets: the partner of an applied swap or of a self
// proposal, n for a proposal that lost its ballot) by plain copies of the device arrays.  Any
// output pointer may be null.
extern "C" int cupim_get(int32_t *phi, int32_t *force, int32_t *score, int32_t *targets) {
    if (!g_open) return -1;
    const size_t rn = (size_t)g_R * g_n;
    std::vector<uint32_t> tmp(rn);
    int rc = 0;
    if (phi) {
        rc = cuda_ok(cudaMemcpy(tmp.data(), g_dev.facility_at_position, rn * 4, cudaMemcpyDeviceToHost));
        if (rc) return rc;
        for (size_t k = 0; k < rn; ++k) phi[k] = (int32_t)tmp[k];
    }
    if (force) rc = cuda_ok(cudaMemcpy(force, g_dev.force_mat, rn * g_n * 4, cudaMemcpyDeviceToHost));
    if (!rc && score) rc = cuda_ok(cudaMemcpy(score, g_dev.replica_score, g_R * 4, cudaMemcpyDeviceToHost));
    if (!rc && targets) {
        rc = cuda_ok(cudaMemcpy(tmp.data(), g_dev.proposed_targets, rn * 4, cudaMemcpyDeviceToHost));
        if (!rc)
            for (size_t k = 0; k < rn; ++k) targets[k] = (int32_t)tmp[k];
    }
    return rc;
}

extern "C" int cupim_close() {
    if (!g_open) return -1;
    g_dev.cu_free();
    g_host.cu_free();
    cudaFree(g_uni);
    g_uni = nullptr;
    g_open = false;
    return cuda_ok(cudaDeviceSynchronize());
}
