// Internal host/device structures of the wvlh library (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace wvlh {

// z-kernel tile: TX_ consecutive x by TY_ rows of columns
constexpr int TX_ = 32;
constexpr int TY_ = 2;
// block sizes of the plane kernels (K1, K3) and of the z-pencil kernel (K2);
// 384 threads give 3 line-segment items per thread on 96-point planes
constexpr int kPlaneThreads = 384;

// CTAs per SM the plane kernels are compiled for (register budget): FP32
// 1024 / 512 / 384 / 256 / 128 threads -> 1 / 2 / 3 / 4 / 8; FP64 (no 1024)
// 512 / 384 / 256 / 128 -> 1 / 1 / 2 / 4.
__host__ __device__ constexpr int plane_ctas_per_sm(bool fp32, int nt)
{
    return fp32 ? (nt >= 1024 ? 1 : nt >= 512 ? 2 : nt >= 384 ? 3 : nt >= 256 ? 4 : 8)
                : (nt >= 384 ? 1 : nt >= 256 ? 2 : 4);
}

// CTA size of the plane kernels, chosen per batch by a small occupancy model:
// a pass has `rows` lines of up to `len` points cut into segments of SEG
// outputs; with nt threads it takes ceil(items / nt) rounds, so the busy
// fraction is items / (rounds nt); the SM holds as many CTAs as registers (the
// compiled count above), shared memory and threads allow.  The expected rate
// is busy x resident threads x ctas / (ctas + 1/2) — the last factor because
// a CTA's barrier waits are covered only by the other resident CTAs; each
// orbital's planes weigh by their work, and the size with the least total cost
// wins (a larger CTA on a tie).
struct PlaneShape {
    long long rows, len, smem_bytes, weight;
};
inline int choose_plane_threads(const std::vector<PlaneShape> &shapes, bool fp32)
{
    const int cand32[5] = {1024, 512, kPlaneThreads, 256, 128};
    const int cand64[4] = {512, kPlaneThreads, 256, 128};
    const int *cand = fp32 ? cand32 : cand64;
    const int ncand = fp32 ? 5 : 4;
    const int seg = fp32 ? 8 : 4;
    double best = 0.0;
    int pick = 0;
    for (int k = 0; k < ncand; ++k) {
        const int nt = cand[k];
        double cost = 0.0;
        for (const PlaneShape &s : shapes) {
            const long long items = s.rows * ((s.len + seg - 1) / seg);
            const long long rounds = (items + nt - 1) / nt;
            const double busy = (double)items / (double)(rounds * nt);
            const long long by_regs = plane_ctas_per_sm(fp32, nt);
            const long long by_smem = (227LL * 1024) / (s.smem_bytes + 1024);
            const long long by_threads = 2048 / nt;
            long long ctas = by_regs < by_smem ? by_regs : by_smem;
            ctas = ctas < by_threads ? ctas : by_threads;
            if (ctas < 1) ctas = 1;
            const double rate = busy * (double)ctas * nt * ((double)ctas / ((double)ctas + 0.5));
            cost += (double)s.weight / rate;
        }
        if (pick == 0 || cost < best * 0.999) {
            best = cost;
            pick = nt;
        }
    }
    return pick;
}
constexpr int kZThreads = 256;

// One localisation region (box + compressed-key tables) as seen by kernels.
// Segments are decoded once on upload from the reference's 1-based keyg/keyv
// (wavelib/un-compress.f90:896-905 arithmetic) into {i0, i2, len, jj0}, with
// jj0 the 0-based compressed position; plane_c/plane_f[i3..i3+1] delimit the
// segments of coarse z-plane i3 (keys are sorted by linear index).
struct LrDev {
    int N[3];
    int per[3];
    int nseg_c, nseg_f;
    int nvctr_c, nvctr_f;
    const int4 *seg_c;
    const int4 *seg_f;
    const int *plane_c;  // N3+1 entries
    const int *plane_f;  // N3+1 entries
    double hgrid[3];     // coarse grid spacing
};

// One orbital job of a batch.
struct OrbDev {
    int lr;
    int pad;
    long long psi;   // element offset of [psi_c | psi_f] in the psi/hpsi arrays
    long long pot;   // element offset of this orbital's potential / density (ISF grid)
    long long sP;    // scratch element offsets: P (G3*F2*F1)
    long long sQ;    //   Q / Z1 (G3*I2*I1)
    long long sZ;    //   Z2 (G3*F2*F1)
    double c;        // shift of (T + c), preconditioner only
    // optional absolute buffers (a batch that spans several owners' arrays);
    // when set they replace base + offset
    const void *in_ptr;
    void *out_ptr;
    const void *pot_ptr;
};

enum FusedMode { MODE_LOCHAM = 0, MODE_LOCDEN = 1, MODE_PRECOND = 2 };

// Host view of an uploaded batch (plan) — owned by the context.
struct Plan {
    int nlr = 0, norb = 0;
    bool all_periodic = false;  // every region periodic in x, y and z
    std::vector<int> lr_N;  // 3*nlr
    std::vector<int> lr_per;
    std::vector<int> orb_lr;
    std::vector<long long> orb_psi;  // element offsets
    long long psi_total = 0;
    long long scratch_elems = 0;     // per "chunk" of all orbitals (full batch)
    // device tables
    LrDev *d_lr = nullptr;
    OrbDev *d_orb = nullptr;
    // work items in runs of one orbital: prefix sums over the orbitals (norb+1
    // entries) of the plane kernels' items (G3 wavelet planes each) and of the
    // z kernels' 32 x 2-column tiles: chain 0 over I1 x I2 (d_pre2), chain 1
    // over F1 x F2 (d_pre2p)
    int *d_pre13 = nullptr;
    int *d_pre2 = nullptr;
    int *d_pre2p = nullptr;
    int n_work13 = 0, n_work2 = 0, n_work2p = 0;
    // density: z-kernel tiles of the I1 x I2 plane, in runs of one chunk
    // (prefix over the chunks) of orbitals that share one density grid (same
    // region, same density key)
    int *d_pred = nullptr;
    int n_workd = 0;
    int nchunk = 0, ngroup = 0;
    int *d_chunk_orb_start = nullptr;    // nchunk + 1 offsets into d_chunk_orbs
    int *d_chunk_orbs = nullptr;
    long long *d_chunk_part = nullptr;   // element offset of each chunk's partial density
    long long part_den_elems = 0;
    int *d_group_chunk_start = nullptr;  // ngroup + 1 chunk ranges
    long long *d_group_rho = nullptr;    // density offset (or address) of each group
    int *d_group_n = nullptr;            // ISF points of each group
    int max_group_n = 0;
    int den_acc = 32;                    // FP64 accumulators per thread of kd_density (32 or 48)
    // per-orbital compressed vector offset / length (preconditioner vector ops)
    long long *d_orb_off = nullptr;
    int *d_orb_len = nullptr;
    int part_stride = 0;           // energy partial slots per orbital
    size_t smem13[2] = {0, 0};     // dynamic smem bytes (float, double) of the two plane buffers
    long long plane_elems = 0;     // elements of plane buffer A (rows x pitch)
    long long planeB_elems = 0;    // elements of buffer B (a plane or a transposed plane)
    int plane_threads[2] = {kPlaneThreads, kPlaneThreads};   // plane-kernel CTA size (float, double)
    int plane_threads_pre[2] = {kPlaneThreads, kPlaneThreads};   // the same for the preconditioner operator
    int z_threads[2] = {kZThreads, kZThreads};       // z-kernel CTA size (FP32: 256, 320 or 384)
    int z_threads_pre[2] = {kZThreads, kZThreads};   // the same for the preconditioner operator
    size_t smem2[2] = {0, 0};
    int pitch_max = 0, rows_max = 0, zlen_max = 0;
    // scratch elements per orbital when every orbital lies in one region (the
    // planes then form regular (x, y, z, orbital) tensors: TMA tiles), else 0;
    // tile_dims = {G3, F1, F2, I1, I2} of that region
    long long orb_scratch = 0;
    long long tile_dims[5] = {0, 0, 0, 0, 0};
    std::vector<void *> owned;     // device allocations to free
};

// Checks the reference's 1-based keys of one region (compression.f90:29-39):
// keyg = (first, last) linear index of each segment in the N[0] x N[1] x N[2]
// box, x fastest, strictly increasing, each segment on one x-line; keyv the
// running 1-based offset of each segment in the compressed vector.  Returns
// WVLH_OK or WVLH_ERR_KEYS; on success nvctr is the number of values.
inline int check_keys(const int *N, int nseg, const int32_t *keyg, const int32_t *keyv, long long *nvctr)
{
    const long long n12 = (long long)N[0] * N[1], ntot = n12 * N[2];
    long long prev_end = 0, cum = 0;
    for (int s = 0; s < nseg; ++s) {
        const long long j0 = keyg[2 * s], j1 = keyg[2 * s + 1];
        if (j0 < 1 || j1 < j0 || j1 > ntot || j0 <= prev_end) return 3;          // WVLH_ERR_KEYS
        if ((j0 - 1) / N[0] != (j1 - 1) / N[0]) return 3;                         // one x-line per segment
        if ((long long)keyv[s] != cum + 1) return 3;
        cum += j1 - j0 + 1;
        prev_end = j1;
    }
    if (nvctr) *nvctr = cum;
    return 0;
}

}  // namespace wvlh
