// nfft_cluster.cu -- instantiation and launch of the cluster-resident
// complex DFT (nfft_cluster.cuh): one transform per thread-block cluster.
#include "nfft_cluster.cuh"
#include "nfft_engine.h"

namespace nfft {

namespace {

struct ClusterEntry {
    int logN, logR1, logC, logT;
    const void* fn;
    size_t smem;
    int ok = -1;   // per-process: -1 unknown, 0 cannot be resident, 1 usable
};

#define NFFT_CLUSTER_ENTRY(R1, R2, LC, LT) \
    ClusterEntry{R1 + R2, R1, LC, LT, (const void*)cluster_fft_kernel<real_t, R1, R2, LC, LT>, cluster_smem_bytes<real_t, R1, R2, LC, LT>()}

// N = 2^14 .. 2^16 (and 2^17 for float): 16 points per thread, column tiles
// of at least 8 lines.
ClusterEntry g_cluster[] = {
    NFFT_CLUSTER_ENTRY(7, 7, 3, 7),
    NFFT_CLUSTER_ENTRY(7, 8, 3, 8),
    NFFT_CLUSTER_ENTRY(8, 8, 4, 8),
#if NFFT_REAL_IS_FLOAT
    NFFT_CLUSTER_ENTRY(8, 9, 4, 9),
#endif
};

std::mutex g_cluster_mu;

ClusterEntry* find_cluster(int logN) {
    for (auto& e : g_cluster)
        if (e.logN == logN) return &e;
    return nullptr;
}

// Attributes (dynamic shared memory, non-portable cluster size) and a
// residency check on the current device; 0 when the cluster cannot run.
int prepare(ClusterEntry& e) {
    std::lock_guard<std::mutex> lk(g_cluster_mu);
    if (e.ok >= 0) return e.ok;
    e.ok = 0;
    if (cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem) != cudaSuccess ||
        cudaFuncSetAttribute(e.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1u << e.logC, 1, 1);
    cfg.blockDim = dim3(1u << e.logT, 1, 1);
    cfg.dynamicSmemBytes = e.smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1u << e.logC;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, e.fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    e.ok = nclusters > 0 ? 1 : 0;
    return e.ok;
}

}  // namespace

bool cluster_available(int logN) {
    // opt-in: on B200 the two-pass kernels measured faster (2^14: 3091 vs 2198 GB/s FP64)
    const char* v = getenv("NOTORIOUS_FFT_CLUSTER");
    if (!v || !atoi(v)) return false;
    ClusterEntry* e = find_cluster(logN);
    return e && prepare(*e) == 1;
}

bool launch_cluster(const PassArgs& a1, const PassArgs& a2, int logN, long long ntransforms, cudaStream_t s) {
    ClusterEntry* e = find_cluster(logN);
    if (!e || prepare(*e) != 1) {
        set_error(6, "no cluster kernel for N = 2^%d", logN);
        return false;
    }
    if (ntransforms <= 0) return true;
    long long blocks = ntransforms << e->logC;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks, 1, 1);
    cfg.blockDim = dim3(1u << e->logT, 1, 1);
    cfg.dynamicSmemBytes = e->smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1u << e->logC;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[] = {(void*)&a1, (void*)&a2, (void*)&ntransforms};
    cudaError_t err = cudaLaunchKernelExC(&cfg, e->fn, args);
    note_launch();
    return cuda_ok(err, "cluster kernel launch");
}

int cluster_logr1(int logN) {
    ClusterEntry* e = find_cluster(logN);
    return e ? e->logR1 : -1;
}

}  // namespace nfft
