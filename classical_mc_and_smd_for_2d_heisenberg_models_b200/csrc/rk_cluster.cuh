// rk_cluster.cuh -- RK4 + energy-correction kernel for one sample spread over
// a thread-block cluster (declarations shared by host and device code).
//
// A sample's N sites are cut into CS contiguous index ranges, one per CTA of
// a cluster.  Each CTA keeps in shared memory the stage values of its own
// sites and of the halo sites (other CTAs' sites that its sites neighbour).
// After computing a stage value a thread stores it locally and pushes it
// into the halo slots of the CTAs that hold a copy (distributed shared
// memory stores).  With async_halo set (the neighbour relation is
// symmetric and a publish fits one mbarrier transaction count), the pushes
// are st.async stores that complete bytes on one of two mbarriers of the
// receiving CTA, and a stage waits for its own halo bytes only; otherwise
// one cluster barrier per stage publishes everything.
//
// Site records are 4-wide vectors (x, y, z, 0), so a neighbour costs one
// vector load; neighbours are local slot numbers packed two per 32-bit word;
// every edge slot e has one coefficient vector J_shell(e) * lambda_shell(e)
// passed as a kernel parameter, which the unrolled edge loop reads as a
// constant operand.  Vacancies (impurities with zero couplings) are handled
// by storing mask * S in the gathered buffers, mask = 1 - impurity flag.
#pragma once

#include "smd_device.cuh"

namespace smd {

constexpr int kMaxEdgeSlots = 20;
constexpr int kMaxClusterCTAs = 16;

struct ClusterParams {
    int N;
    int CS;                // CTAs per sample
    int n_own_max;         // largest own range
    int n_loc_max;         // largest own + halo count
    int pmax;              // push entries per own site
    int ZT;                // edge slots (padded to the kernel's template value)
    int energy_from_field; // must be 1 (host routes other lattices elsewhere)
    int async_halo;        // halo pushes complete transactions on the receiver's mbarriers
    double h;
    float hf;
    double coef64[kMaxEdgeSlots][3];
    float coef32[kMaxEdgeSlots][3];
    const int *own_base;   // [CS]
    const int *own_cnt;    // [CS]
    const int *halo_cnt;   // [CS]
    const int *halo_gid;   // [CS][n_loc_max]
    const uint32_t *idx;   // [CS][ZT/2][n_own_max] packed local slots
    const int *push;       // [CS][pmax][n_own_max] (rank << 16 | slot) or -1
};

// Batched form: one persistent launch integrates the samples of several
// lattices (slots), each with its own partition, coefficients and buffers.
// Clusters of CSH CTAs take work items (slot, first sample) from a device
// queue; a slot whose partition has CS <= CSH CTAs (CS dividing CSH) runs
// CSH / CS samples per item, one per group of CS CTAs.  The item list is
// ordered by the host (largest per-CTA work first).
constexpr int kMaxBatchSlots = 24;

struct BatchSlot {
    ClusterParams P;   // partition of the slot's lattice (P.CS CTAs per sample)
    RKJob J;           // the slot's buffers and record range for this launch
};

struct BatchParams {
    int n_slots;
    int n_items;
    const int2 *items;   // [n_items]: (slot, first sample of the item)
    int *queue;          // next item; zero before the launch
    BatchSlot slot[kMaxBatchSlots];
};

// Launch of the persistent batch kernel: nclusters clusters of csh CTAs of
// `threads` threads each; zt = edge slots of every slot's tables.
cudaError_t launch_rk_batch(const BatchParams &B, int precision, int spt, int zt, int threads, int csh,
                            int nclusters, size_t smem, cudaStream_t st);
// Clusters of the batch kernel that fit the device at once (0 if none).
int rk_batch_max_clusters(int precision, int spt, int zt, int threads, int csh, size_t smem);
// Threads per CTA of the batch kernel for a sites-per-thread value.
int rk_batch_threads(int precision, int spt);

size_t rk_cluster_smem(const ClusterParams &P, int precision);
// qss[s][r] = r == 0 ? 1 : (1 / N) * sum over the CS partials of record r,
// summed in rank order (the order of the in-cluster reduction)
cudaError_t launch_qss_from_parts(const double *qpart, int W, int n_rec, int CS, int N, double *qss,
                                  cudaStream_t st);
int rk_cluster_maxt(int precision, int spt);
cudaError_t launch_rk_cluster(const ClusterParams &P, const RKJob &J, int precision, int spt,
                              int threads, cudaStream_t st);

}  // namespace smd
