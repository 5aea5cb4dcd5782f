// nbsearch.cu — cell-grid / neighbour-list build.
//
// Replaces NeighborLists::updateNlists (code/LIMA_ENGINE/src/Neighborlists.cuh:294-317)
// and its O(N_c^2) compound test (:139-229) with an O(N) column-cluster build:
//   1. k_bin            atom -> column of an x-y grid (wrapped positions)
//   2. k_scan_columns   per-system exclusive scans: atom and cluster offsets
//   3. k_scatter        atoms -> column lists (unordered)
//   4. k_sort_columns   deterministic order inside a column: (z, atom index),
//                       then in each cluster of 8 the atoms with LJ first
//   5. k_gather_slots   state permuted into the new slot order
//   6. k_finish_slots   slot_of map, permuted velocity state
//   7. k_bbox           per-cluster bounding boxes
//   8. k_pairsearch     half list of cluster pairs within cutoff+skin, stored
//                       as rows: one per j-atom with a non-empty 8-bit mask of
//                       the i-atoms it meets (padding and exclusions taken out;
//                       a cluster with itself keeps i<j unshifted and one image
//                       of each +/- pair of its own periodic images) and the
//                       pair's periodic image.
// The result is bit-identical run to run: every ordering is fixed by keys,
// never by atomic arrival order.
#include "engine.h"
#include "packed.cuh"

namespace lima {

// Adds one to counter[key] for every lane with key >= 0, one atomic per group of
// lanes sharing a key; returns the lane's place within its group's block.
__device__ __forceinline__ int warp_add_counts(int* counter, int key) {
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader && key >= 0) base = atomicAdd(counter + key, __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// One thread per atom (a build from new input) or per slot (a rebuild from the
// engine's own slots: the atoms of a warp then mostly share a column, and the
// column counts take one atomic per column and warp).
__global__ void k_bin(DevState st, int from_input) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int a = -1, s = -1;
    if (from_input) {
        if (t < st.n_atoms) a = t;
    } else if (t < st.n_slots) {
        s = t;
        a = st.orig[t];
    }
    int col = -1;
    if (a >= 0) {
        const SysDesc& sd = st.sys[st.atom_sys[a]];
        double p[3];
        if (from_input) {
            p[0] = st.in_pos[3 * a];
            p[1] = st.in_pos[3 * a + 1];
            p[2] = st.in_pos[3 * a + 2];
        } else {
            p[0] = st.px[s];
            p[1] = st.py[s];
            p[2] = st.pz[s];
        }
        for (int d = 0; d < 3; ++d) {
            double x = p[d];
            if (st.periodic) {   // wrapped into the box; without a boundary condition kept as is
                const double L = sd.box[d];
                x -= L * floor(x / L);
                if (x >= L) x -= L;
                if (x < 0.0) x = 0.0;
            }
            p[d] = x;
            st.in_pos[3 * a + d] = x;
        }
        // column of the position; one outside the box (no boundary condition) is
        // binned at the box's edge
        const int cx = (int)fmin(fmax(p[0] * sd.ncol_x / sd.box[0], 0.0), (double)(sd.ncol_x - 1));
        const int cy = (int)fmin(fmax(p[1] * sd.ncol_y / sd.box[1], 0.0), (double)(sd.ncol_y - 1));
        col = sd.col_off + cx + sd.ncol_x * cy;
        st.col_of_atom[a] = col;
        st.z_of_atom[a] = (float)p[2];
    }
    warp_add_counts(st.col_count, col);
}

// one CTA per system; Hillis-Steele block scan over chunks of columns
__global__ void k_scan_columns(DevState st) {
    const int s = blockIdx.x;
    const SysDesc sd = st.sys[s];
    const int ncol = sd.ncol_x * sd.ncol_y;
    __shared__ int sa[1024], sc[1024];
    __shared__ int carry_a, carry_c;
    const int tid = threadIdx.x;
    if (tid == 0) carry_a = carry_c = 0;
    __syncthreads();
    for (int base = 0; base < ncol; base += blockDim.x) {
        const int i = base + tid;
        const int cnt = i < ncol ? st.col_count[sd.col_off + i] : 0;
        const int ncl = (cnt + CLUSTER - 1) / CLUSTER;
        sa[tid] = cnt;
        sc[tid] = ncl;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            const int va = tid >= o ? sa[tid - o] : 0;
            const int vc = tid >= o ? sc[tid - o] : 0;
            __syncthreads();
            sa[tid] += va;
            sc[tid] += vc;
            __syncthreads();
        }
        if (i < ncol) {
            // clusters past the system's capacity are cut (the overflow flag makes
            // the host reject the build), so that no reader leaves the system's slots
            const int c0 = min(carry_c + sc[tid] - ncl, sd.max_clusters);
            st.col_atom_start[sd.col_off + i] = carry_a + sa[tid] - cnt;
            st.col_cl_start[sd.col_off + i] = sd.cluster_cap_off + c0;
            st.col_ncl[sd.col_off + i] = min(ncl, sd.max_clusters - c0);
        }
        __syncthreads();
        if (tid == blockDim.x - 1) {
            carry_a += sa[tid];
            carry_c += sc[tid];
        }
        __syncthreads();
    }
    if (tid == 0) {
        st.sys_nclusters[s] = min(carry_c, sd.max_clusters);
        if (carry_c > sd.max_clusters) atomicOr(st.status, ST_COLUMN_OVERFLOW);
    }
}

// atoms -> column lists, in the same thread order as k_bin (the order within a
// column is fixed afterwards by the sort)
__global__ void k_scatter(DevState st, int from_input) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int a = -1;
    if (from_input) {
        if (t < st.n_atoms) a = t;
    } else if (t < st.n_slots) {
        a = st.orig[t];
    }
    const int col = a >= 0 ? st.col_of_atom[a] : -1;
    const int k = warp_add_counts(st.col_fill, col);
    if (a >= 0) {
        const int off = st.sys[st.atom_sys[a]].atom_off;
        st.col_list[off + st.col_atom_start[col] + k] = a;
    }
}

// One CTA per column: the column's atoms sorted by the unique key (z bits, atom
// index) with a bitonic network in shared memory over the next power of two of
// the column's count; padding keys are all ones and sort last.  The keys are
// unique, so the order is the one a rank count gives, whatever the network.
__global__ void k_sort_columns(DevState st, const int* col_sys) {
    extern __shared__ unsigned long long keys[];
    const int col = blockIdx.x;
    const int n_all = st.col_count[col];
    const int n = min(n_all, st.col_cap);
    const int off = st.sys[col_sys[col]].atom_off + st.col_atom_start[col];
    const int slot0 = st.col_cl_start[col] * CLUSTER;
    const int padded = st.col_ncl[col] * CLUSTER;
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        unsigned long long k = ~0ull;
        if (i < n) {
            const int a = st.col_list[off + i];
            // z bits made order-preserving for negative z too (no boundary condition)
            unsigned z = __float_as_uint(st.z_of_atom[a]);
            z ^= (z >> 31) ? 0xffffffffu : 0x80000000u;
            k = ((unsigned long long)z << 32) | (unsigned)a;
        }
        keys[i] = k;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            // pair t compares elements i and i + j, i with bit j clear
            for (int t = threadIdx.x; t < (m >> 1); t += blockDim.x) {
                const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const unsigned long long a = keys[i], b = keys[i + j];
                if ((a > b) == ((i & k) == 0)) {
                    keys[i] = b;
                    keys[i + j] = a;
                }
            }
            __syncthreads();
        }
    // Clusters are runs of 8 ranks; inside each, the atoms with LJ (eps != 0) take
    // the first slots, each part in z order (so the pair kernel can leave the LJ
    // arithmetic out for the cluster's trailing LJ-free atom pairs: in water the
    // hydrogens).  The cluster's atom set, and so its box, is that of the z order.
    // Ranks past the column's cluster range are cut (overflow, flagged below).
    for (int g = threadIdx.x; g * CLUSTER < padded; g += blockDim.x) {
        int a[CLUSTER];
        unsigned lj = 0u;
#pragma unroll
        for (int r = 0; r < CLUSTER; ++r) {
            const int rr = g * CLUSTER + r;
            a[r] = rr < n ? (int)(keys[rr] & 0xffffffffu) : -1;
            if (a[r] >= 0 && st.ljp_atom[a[r]].y != 0.f) lj |= 1u << r;
        }
        int out = 0;
#pragma unroll
        for (int r = 0; r < CLUSTER; ++r)
            if ((lj >> r) & 1u) st.new_orig[slot0 + g * CLUSTER + out++] = a[r];
#pragma unroll
        for (int r = 0; r < CLUSTER; ++r)   // then the other atoms, padding (-1) last
            if (!((lj >> r) & 1u)) st.new_orig[slot0 + g * CLUSTER + out++] = a[r];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n_all > st.col_cap) atomicOr(st.status, ST_COLUMN_OVERFLOW);
        st.col_count[col] = 0;
        st.col_fill[col] = 0;
    }
}

__global__ void k_gather_slots(DevState st, int from_input) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots) return;
    const int c = s / CLUSTER;
    const int sysi = st.cluster_sys[c];
    const SysDesc& sd = st.sys[sysi];
    const int local = c - sd.cluster_cap_off;
    const int a = local < st.sys_nclusters[sysi] ? st.new_orig[s] : -1;
    if (a >= 0) {
        const double x = st.in_pos[3 * a], y = st.in_pos[3 * a + 1], z = st.in_pos[3 * a + 2];
        st.px[s] = x;
        st.py[s] = y;
        st.pz[s] = z;
        st.xyzq[s] = make_float4((float)x, (float)y, (float)z, st.q[a]);
        st.xyz_ref[s] = st.xyzq[s];
        st.ljp[s] = st.ljp_atom[a];
        const float im = st.inv_mass[a];
        if (from_input) {
            st.tvel[s] = make_float4(st.in_vel[3 * a], st.in_vel[3 * a + 1], st.in_vel[3 * a + 2], im);
            st.tfprev[s] = make_float4(0.f, 0.f, 0.f, 0.f);
            st.tadam_m[s] = make_float4(0.f, 0.f, 0.f, 0.f);
            st.tadam_v[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            const int old = st.slot_of[a];
            float4 v = st.vel[old];
            v.w = im;
            st.tvel[s] = v;
            st.tfprev[s] = st.fprev[old];
            st.tadam_m[s] = st.adam_m[old];
            st.tadam_v[s] = st.adam_v[old];
        }
    } else {
        st.px[s] = 0.0;
        st.py[s] = 0.0;
        st.pz[s] = 0.0;
        st.xyzq[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        st.ljp[s] = make_float2(0.f, 0.f);
        st.tvel[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        st.tfprev[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        st.tadam_m[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        st.tadam_v[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    st.orig[s] = a;
    st.slot_mol[s] = a >= 0 ? st.mol[a] : -1;
}

__global__ void k_finish_slots(DevState st) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots) return;
    st.vel[s] = st.tvel[s];
    st.fprev[s] = st.tfprev[s];
    st.adam_m[s] = st.tadam_m[s];
    st.adam_v[s] = st.tadam_v[s];
    const int a = st.orig[s];
    if (a >= 0) st.slot_of[a] = s;
}

__global__ void k_bbox(DevState st) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= st.n_clusters) return;
    float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
    bool first = true;
    unsigned long long sig = 0ull;
    for (int k = 0; k < CLUSTER; ++k) {
        const int s = c * CLUSTER + k;
        if (st.orig[s] < 0) continue;
        sig |= 1ull << (st.slot_mol[s] & 63);
        const float4 p = st.xyzq[s];
        if (first) {
            lo = hi = p;
            first = false;
        } else {
            lo.x = fminf(lo.x, p.x);
            lo.y = fminf(lo.y, p.y);
            lo.z = fminf(lo.z, p.z);
            hi.x = fmaxf(hi.x, p.x);
            hi.y = fmaxf(hi.y, p.y);
            hi.z = fmaxf(hi.z, p.z);
        }
    }
    lo.w = first ? 0.f : 1.f;  // w = 1 marks a populated cluster
    st.bb_lo[c] = lo;
    st.bb_hi[c] = hi;
    st.bb_molsig[c] = sig;
}

__device__ __forceinline__ bool excluded(const DevState& st, int ai, int aj, int eb, int ee) {
    for (int k = eb; k < ee; ++k)
        if (st.excl_idx[k] == aj) return true;
    return false;
}

// One warp per i-cluster, in two phases that alternate through the column
// window:
//   1. candidate search: the window's columns are scanned 32 at a time (one per
//      lane: periodic shift, clusters of the half list) and their clusters taken
//      32 at a time (one per lane) and tested against the i-cluster's extent for
//      each periodic image in range; every (cluster, image) in range is
//      appended, in lane order, to a per-warp queue in shared memory;
//   2. rows: whenever 32 candidates are queued, four at a time are turned into
//      rows, one lane per (candidate, j-atom) testing its j-atom against the
//      eight i-atoms (held in registers); the non-empty rows are appended in
//      lane order.
// Instruction count, not memory, bounds this kernel.  The list order is fixed
// by the column, cluster, lane and image order, so the list is identical run to
// run.
constexpr int PS_WARPS = 4;
constexpr int PS_QCAP = 32 + 32 * 27;   // a full batch left over + one column batch with every shift

// SPLIT (a small system's engine, as in the pair kernel): the warps of an
// i-cluster share its window, each taking a contiguous slice of the virtual
// columns; their rows, concatenated in slice order, are the rows one warp would
// have produced (k_pairsearch_concat).
template <bool SPLIT>
__global__ void __launch_bounds__(PS_WARPS * 32, 1) k_pairsearch(DevState st, float rlist) {
    __shared__ int q[PS_WARPS][PS_QCAP];
    __shared__ int s_mi[PS_WARPS][CLUSTER], s_ai[PS_WARPS][CLUSTER];
    __shared__ int s_end[PS_WARPS][32], s_js[PS_WARPS][32], s_sh[PS_WARPS][32];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (warp >= (SPLIT ? st.nb_warps : st.n_clusters)) return;
    int ci = warp, sysi, parts = 1, part = 0;
    if (!SPLIT) {
        sysi = st.cluster_sys[ci];
    } else {
        sysi = 0;
        for (int hi = st.n_sys - 1; sysi < hi;) {
            const int mid = (sysi + hi + 1) >> 1;
            if (st.nb_warp_off[mid] <= warp) sysi = mid;
            else hi = mid - 1;
        }
        parts = max(1, st.sys[sysi].nb_parts);
        const int lw = warp - st.nb_warp_off[sysi], lp = __ffs(parts) - 1;
        ci = st.sys[sysi].cluster_cap_off + (lw >> lp);
        part = lw & (parts - 1);
    }
    const SysDesc& sd = st.sys[sysi];
    const int local = ci - sd.cluster_cap_off;
    if (local >= st.sys_nclusters[sysi]) {
        if (lane == 0) {
            if (SPLIT) st.ps_stage_count[warp] = 0;
            else st.pl_count[ci] = 0;
        }
        return;
    }
    const float4 ilo = st.bb_lo[ci], ihi = st.bb_hi[ci];
    const float ic[3] = {0.5f * (ilo.x + ihi.x), 0.5f * (ilo.y + ihi.y), 0.5f * (ilo.z + ihi.z)};
    const float ie[3] = {0.5f * (ihi.x - ilo.x), 0.5f * (ihi.y - ilo.y), 0.5f * (ihi.z - ilo.z)};
    const float L[3] = {sd.boxf[0], sd.boxf[1], sd.boxf[2]};
    const float R = rlist, R2 = rlist * rlist;

    const unsigned long long isig = st.bb_molsig[ci];
    // the eight i-atoms in every lane's registers; a padding i-atom is moved far
    // away so that no distance test passes for it
    float xi[CLUSTER], yi[CLUSTER], zi[CLUSTER];
#pragma unroll
    for (int a = 0; a < CLUSTER; ++a) {
        const int s = ci * CLUSTER + a;
        const float4 x = st.xyzq[s];
        const bool real = st.orig[s] >= 0;
        xi[a] = real ? x.x : 1e30f;
        yi[a] = real ? x.y : 1e30f;
        zi[a] = real ? x.z : 1e30f;
    }
    // molecule ids and atom indices of the i-atoms, for the rare exclusion test
    if (lane < CLUSTER) {
        s_mi[wib][lane] = st.slot_mol[ci * CLUSTER + lane];
        s_ai[wib][lane] = st.orig[ci * CLUSTER + lane];
    }
    __syncwarp();

    // column window (every column visited once even when the window wraps).
    // When it does not cover a whole row of columns, each column in it is met
    // once at a known unwrapped position, which fixes the x and y periodic
    // shift of its clusters: only the three z shifts remain to test.
    // Otherwise every one of the 27 shifts is tested.
    int cx0 = (int)floorf((ilo.x - R) / sd.col_w[0]);
    int nx = (int)floorf((ihi.x + R) / sd.col_w[0]) - cx0 + 1;
    bool fixed_xy = true;
    if (nx >= sd.ncol_x) {
        cx0 = 0;
        nx = sd.ncol_x;
        fixed_xy = false;
    }
    int cy0 = (int)floorf((ilo.y - R) / sd.col_w[1]);
    int ny = (int)floorf((ihi.y + R) / sd.col_w[1]) - cy0 + 1;
    if (ny >= sd.ncol_y) {
        cy0 = 0;
        ny = sd.ncol_y;
        fixed_xy = false;
    }
    if (!st.periodic) {
        // no images: the columns the extent reaches, clamped to the grid (atoms
        // outside the box are binned in its edge columns), each met once unshifted
        auto col_of = [](float v, int n) { return (int)fminf(fmaxf(v, 0.f), (float)(n - 1)); };
        cx0 = col_of(floorf((ilo.x - R) / sd.col_w[0]), sd.ncol_x);
        nx = col_of(floorf((ihi.x + R) / sd.col_w[0]), sd.ncol_x) - cx0 + 1;
        cy0 = col_of(floorf((ilo.y - R) / sd.col_w[1]), sd.ncol_y);
        ny = col_of(floorf((ihi.y + R) / sd.col_w[1]), sd.ncol_y) - cy0 + 1;
        fixed_xy = true;
    }

    const int cap = st.pl_cap;
    int count = 0;
    int2* const rows_out = SPLIT ? st.ps_stage : st.pl_row;
    const size_t base_out = (size_t)(SPLIT ? warp : ci) * cap;

    // rows of the queued candidates q[head .. head + nb): four candidates per
    // pass, one lane per (candidate, j-atom), each lane testing its j-atom against
    // the 8 i-atoms; rows leave in candidate order, then j-atom order
    auto build_masks = [&](int head, int nb) {
        const int jj = lane & 7;
#pragma unroll 1
        for (int c0 = 0; c0 < nb; c0 += 4) {
            const int c = c0 + (lane >> 3);
            unsigned m8 = 0u;
            int sj = 0, code = 0;
            if (c < nb) {
                const int ent = q[wib][head + c];
                const int jc = ent & ((1 << JCLUSTER_BITS) - 1);
                code = (int)((unsigned)ent >> JCLUSTER_BITS);
                const int3 sh = decode_shift(code);
                sj = jc * CLUSTER + jj;
                const int mj = st.slot_mol[sj];
                const float4 xj = st.xyzq[sj];
                const float jx = xj.x + sh.x * L[0], jy = xj.y + sh.y * L[1], jz = xj.z + sh.z * L[2];
#pragma unroll
                for (int ii = 0; ii < CLUSTER; ++ii) {
                    const float dx = jx - xi[ii], dy = jy - yi[ii], dz = jz - zi[ii];
                    if (dx * dx + dy * dy + dz * dz < R2) m8 |= 1u << ii;
                }
                if (mj < 0) m8 = 0u;   // padding slot
                // pairs within one molecule: drop the excluded ones (only when the
                // clusters' molecule signatures meet; then the exclusion lists decide)
                if (m8 != 0u && (isig & st.bb_molsig[jc]) != 0ull) {
                    const int aj = st.orig[sj];
#pragma unroll 1
                    for (int ii = 0; ii < CLUSTER; ++ii) {
                        if (((m8 >> ii) & 1u) && s_mi[wib][ii] == mj) {
                            const int ai = s_ai[wib][ii];
                            if (excluded(st, ai, aj, st.excl_off[ai], st.excl_off[ai + 1])) m8 &= ~(1u << ii);
                        }
                    }
                }
                // the i-cluster with itself counts each pair once: unshifted, ii < jj;
                // against its own periodic image (code > 13 only: the image -s of a
                // pair under shift s is the same pair), every ii other than jj.  An
                // own image is in range only when the cluster spans most of the box
                // (a sparse system), never for an atom with itself (box > 2 r_list)
                if (jc == ci) m8 &= code == 13 ? (1u << jj) - 1u : ~(1u << jj);
            }
            const unsigned has = __ballot_sync(0xffffffffu, m8 != 0u);
            const int pos = count + __popc(has & ((1u << lane) - 1u));
            if (m8 != 0u && pos < cap) {
                const int img = code % 3 | ((code / 3) % 3) << 2 | (code / 9) << 4;
                rows_out[base_out + pos] = make_int2(sj, (int)m8 | (img << ROW_SHIFT_BIT));
            }
            count += __popc(has);
        }
    };

    // Walk of the window's columns, flattened.  The window is taken 32 columns
    // at a time: one pass gives each lane a column (its periodic shift and the
    // clusters it holds for ci's half list, those >= ci) and a scan of their
    // counts; the warp then takes the concatenated clusters 32 at a time, each lane
    // finding its column by binary search over the scan.  Candidates are queued in
    // column, cluster, lane and shift order; full batches of 32 are turned into
    // rows, and after the walk whatever remains.
    // With the x and y shifts fixed, the window is also cut in z: a column's
    // atoms are sorted by z, so its clusters' lower and upper z bounds both rise
    // with the cluster index, and the clusters whose z extent (under a z shift)
    // reaches the i-cluster's z range widened by r_list form one index range,
    // found by two binary searches.  The window is then walked as virtual
    // columns (column, z shift): only the unshifted image, plus the shift down
    // or up when the range crosses the bottom or top of the box.  The range is
    // widened by 1e-4 nm so that it holds every cluster the extent test below
    // could pass; that test still decides.
    const bool zcut = fixed_xy;
    int zs1 = 0, zs2 = 0, nsz = 1;   // z shifts of the second and third virtual column
    float zr_lo = 0.f, zr_hi = 0.f;
    if (zcut) {
        zr_lo = ilo.z - R - 1e-4f;
        zr_hi = ihi.z + R + 1e-4f;
        if (st.periodic) {
            const bool down = zr_lo < 0.f, up = zr_hi >= L[2];
            nsz = 1 + (down ? 1 : 0) + (up ? 1 : 0);
            zs1 = down ? -1 : 1;
            zs2 = 1;
        }
    }
    int qn = 0;
    const int nwin = (nx > 0 && ny > 0) ? nx * ny * nsz : 0;
    // this warp's slice of the virtual columns
    const int v_begin = SPLIT ? (int)((long long)nwin * part / parts) : 0;
    const int v_end = SPLIT ? (int)((long long)nwin * (part + 1) / parts) : nwin;
    for (int w0 = v_begin; w0 < v_end; w0 += 32) {
        const int v = w0 + lane;
        const int w = v / nsz, vz = v - w * nsz;
        int cnt = 0, jstart = 0, shc = 5 | (1 << 4);   // shc: (sx + 1) | (sy + 1) << 2 | (sz + 1) << 4
        const int wy = w / nx, wx = w - wy * nx;
        const int ux = cx0 + wx, uy = cy0 + wy;   // unwrapped column
        // a window narrower than the grid sits within one period of it; a column
        // further out (not met in practice) is left out rather than misaddressed
        if (v < v_end && ux >= -sd.ncol_x && ux < 2 * sd.ncol_x && uy >= -sd.ncol_y && uy < 2 * sd.ncol_y) {
            const int sxc = ux < 0 ? -1 : (ux >= sd.ncol_x ? 1 : 0);
            const int syc = uy < 0 ? -1 : (uy >= sd.ncol_y ? 1 : 0);
            const int col = sd.col_off + (ux - sxc * sd.ncol_x) + sd.ncol_x * (uy - syc * sd.ncol_y);
            const int j0 = st.col_cl_start[col], nj = st.col_ncl[col];
            // clusters are numbered in column order: those before ci are in
            // their own half lists
            jstart = max(j0, ci);
            int jend = j0 + nj;
            const int szc = vz == 0 ? 0 : (vz == 1 ? zs1 : zs2);
            if (zcut && jstart < jend) {
                // first cluster whose top reaches the range, first whose bottom is past it
                const float zl = zr_lo - szc * L[2], zh = zr_hi - szc * L[2];
                int a0 = jstart, a1 = jend, b0 = jstart, b1 = jend;
                while (a0 < a1 || b0 < b1) {
                    const int am = (a0 + a1) >> 1, bm = (b0 + b1) >> 1;
                    const float hz = a0 < a1 ? st.bb_hi[am].z : 0.f;
                    const float lz = b0 < b1 ? st.bb_lo[bm].z : 0.f;
                    if (a0 < a1) {
                        if (hz < zl) a0 = am + 1;
                        else a1 = am;
                    }
                    if (b0 < b1) {
                        if (lz <= zh) b0 = bm + 1;
                        else b1 = bm;
                    }
                }
                jstart = a0;
                jend = max(a0, b0);
            }
            cnt = max(0, jend - jstart);
            shc = (sxc + 1) | ((syc + 1) << 2) | ((szc + 1) << 4);
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_end[wib][lane] = incl;
        s_js[wib][lane] = jstart;
        s_sh[wib][lane] = shc;
        const int tot = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();
        for (int t0 = 0; t0 < tot; t0 += 32) {
            const int t = t0 + lane;
            unsigned shifts = 0u;  // bit k set: shift code k is in range
            int j = 0;
            if (t < tot) {
                // the lane's column: the first whose running count exceeds t
                int lo = 0, hi = 31;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (s_end[wib][mid] > t) hi = mid;
                    else lo = mid + 1;
                }
                j = s_js[wib][lo] + t - (lo ? s_end[wib][lo - 1] : 0);
                const int sx_col = (s_sh[wib][lo] & 3) - 1, sy_col = ((s_sh[wib][lo] >> 2) & 3) - 1;
                const int sz_col = (s_sh[wib][lo] >> 4) - 1;
                const float4 jlo = st.bb_lo[j], jhi = st.bb_hi[j];
                const float jc[3] = {0.5f * (jlo.x + jhi.x), 0.5f * (jlo.y + jhi.y), 0.5f * (jlo.z + jhi.z)};
                const float je[3] = {0.5f * (jhi.x - jlo.x), 0.5f * (jhi.y - jlo.y), 0.5f * (jhi.z - jlo.z)};
                if (jlo.w == 0.f) {
                    // empty cluster: nothing to pair with
                } else if (fixed_xy) {
                    const float gx = fmaxf(fabsf(jc[0] + sx_col * L[0] - ic[0]) - ie[0] - je[0], 0.f);
                    const float gy = fmaxf(fabsf(jc[1] + sy_col * L[1] - ic[1]) - ie[1] - je[1], 0.f);
                    const float gxy = gx * gx + gy * gy;
                    if (gxy < R2) {
                        // the virtual column's z shift
                        const int code = (sx_col + 1) + 3 * (sy_col + 1) + 9 * (sz_col + 1);
                        const float gz = fmaxf(fabsf(jc[2] + sz_col * L[2] - ic[2]) - ie[2] - je[2], 0.f);
                        // own images: one of each +/- pair
                        if (!(j == ci && code < 13) && gxy + gz * gz < R2) shifts |= 1u << code;
                    }
                } else {
                    float g2[3][3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
#pragma unroll
                        for (int sh = -1; sh <= 1; ++sh) {
                            const float dd = fabsf(jc[d] + sh * L[d] - ic[d]) - ie[d] - je[d];
                            const float g = fmaxf(dd, 0.f);
                            g2[d][sh + 1] = g * g;
                        }
                    }
#pragma unroll 1
                    for (int code = 0; code < 27; ++code) {
                        if (j == ci && code < 13) continue;   // own images: one of each +/- pair
                        const int sx = code % 3, sy = (code / 3) % 3, sz = code / 9;
                        const float gxs = sx == 0 ? g2[0][0] : (sx == 1 ? g2[0][1] : g2[0][2]);
                        const float gys = sy == 0 ? g2[1][0] : (sy == 1 ? g2[1][1] : g2[1][2]);
                        const float gzs = sz == 0 ? g2[2][0] : (sz == 1 ? g2[2][1] : g2[2][2]);
                        if (gxs + gys + gzs < R2) shifts |= 1u << code;
                    }
                }
            }
            if (!st.periodic) shifts &= 1u << 13;   // the unshifted image only
            // append (cluster, shift) candidates in lane order, then shift order
            const int c = __popc(shifts);
            int inc2 = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, inc2, o);
                if (lane >= o) inc2 += v;
            }
            const int added = __shfl_sync(0xffffffffu, inc2, 31);
            int wq = qn + inc2 - c;
            while (shifts) {
                const int code = __ffs(shifts) - 1;
                shifts &= shifts - 1u;
                q[wib][wq++] = j | (code << JCLUSTER_BITS);
            }
            qn += added;
            __syncwarp();
            int head = 0;
            while (qn - head >= 32) {
                build_masks(head, 32);
                head += 32;
            }
            if (head > 0) {
                // move the remainder (< 32) to the front of the queue
                const int rem = qn - head;
                const int v = lane < rem ? q[wib][head + lane] : 0;
                __syncwarp();
                if (lane < rem) q[wib][lane] = v;
                qn = rem;
            }
            __syncwarp();
        }
        __syncwarp();   // s_end etc. are rewritten by the next 32 columns
    }
    if (qn > 0) build_masks(0, qn);
    if (lane == 0) {
        if (SPLIT) {
            st.ps_stage_count[warp] = count;   // may pass cap: the concatenation flags it
        } else {
            st.pl_count[ci] = min(count, cap);
            if (count > cap) {
                atomicOr(st.status, ST_PAIRLIST_OVERFLOW);
                atomicMax(st.status + 1, (unsigned)count);   // the capacity this build needed
            }
        }
    }
}

// The split search's rows of each i-cluster, part after part, into pl_row: one
// warp per cluster.  A list longer than the capacity is cut there and flagged
// with the length it needs, as the unsplit search does.
__global__ void k_pairsearch_concat(DevState st) {
    const int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (ci >= st.n_clusters) return;
    const int sysi = st.cluster_sys[ci];
    const SysDesc& sd = st.sys[sysi];
    const int parts = max(1, sd.nb_parts);
    const int w0 = st.nb_warp_off[sysi] + (ci - sd.cluster_cap_off) * parts;
    const int cap = st.pl_cap;
    int2* out = st.pl_row + (size_t)ci * cap;
    int total = 0;
    for (int pp = 0; pp < parts; ++pp) {
        const int c = st.ps_stage_count[w0 + pp];
        const int2* in = st.ps_stage + (size_t)(w0 + pp) * cap;
        const int nc = min(c, cap);
        for (int k = lane; k < nc && total + k < cap; k += 32) out[total + k] = in[k];
        total += c;
    }
    if (lane == 0) {
        st.pl_count[ci] = min(total, cap);
        if (total > cap) {
            atomicOr(st.status, ST_PAIRLIST_OVERFLOW);
            atomicMax(st.status + 1, (unsigned)total);
        }
    }
}

// Dynamic pruning: the inner list holds the rows of the outer list (built at
// rc + skin every nstlist steps) whose j-atom is within rin of at least one
// i-atom now, with the mask cut to those i-atoms, in the outer list's order.
// The pair kernels walk it for the next few steps: rin - rc covers the moves
// of those steps as the skin covers the whole list period, and each pruned row
// spares the pair kernel its 8 evaluations (on the 100k-atom water box about
// 11 % of the rows at rc + 0.05 nm).  One warp per i-cluster; the kept rows of
// each chunk of 32 are compacted with a ballot, so the order is fixed.
// Four rows per lane are in flight at once (their row and j-atom loads issue
// together); the kept rows are written in list order, so the inner list is the
// same whatever the launch shape.  The distance tests are branch-free and take
// the i-atoms two at a time in packed FP32, (2 ip, 2 ip + 1) as the mask bits.
constexpr int PRUNE_ROWS_PER_LANE = 4;

__global__ void __launch_bounds__(256) k_prune_rows(DevState st, float rin2) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= st.n_clusters) return;
    const int ci = warp;
    const int n = min(st.pl_count[ci], st.pl_cap);
    const size_t base = (size_t)ci * st.pl_cap;
    const int sysi = st.cluster_sys[ci];
    const float Lx = st.sys[sysi].boxf[0], Ly = st.sys[sysi].boxf[1], Lz = st.sys[sysi].boxf[2];
    f2p xi[CLUSTER / 2], yi[CLUSTER / 2], zi[CLUSTER / 2];
#pragma unroll
    for (int ip = 0; ip < CLUSTER / 2; ++ip) {
        const float4 a = st.xyzq[ci * CLUSTER + 2 * ip], b = st.xyzq[ci * CLUSTER + 2 * ip + 1];
        xi[ip] = pk2(a.x, b.x), yi[ip] = pk2(a.y, b.y), zi[ip] = pk2(a.z, b.z);
    }
    const unsigned below = (1u << lane) - 1u;
    int out = 0;
    constexpr int U = PRUNE_ROWS_PER_LANE;
    for (int k0 = 0; k0 < n; k0 += 32 * U) {
        int2 row[U];
        float4 xj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u * 32 + lane;
            row[u] = k < n ? st.pl_row[base + k] : make_int2(0, 0);   // mask 0: never kept
        }
#pragma unroll
        for (int u = 0; u < U; ++u) xj[u] = st.xyzq[row[u].x];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const unsigned img = (unsigned)row[u].y >> ROW_SHIFT_BIT;
            const f2p jx = splat2(xj[u].x + fmaf((float)(img & 3u), Lx, -Lx));
            const f2p jy = splat2(xj[u].y + fmaf((float)((img >> 2) & 3u), Ly, -Ly));
            const f2p jz = splat2(xj[u].z + fmaf((float)(img >> 4), Lz, -Lz));
            unsigned bits = 0u;
#pragma unroll
            for (int ip = 0; ip < CLUSTER / 2; ++ip) {
                const f2p dx = sub2(jx, xi[ip]), dy = sub2(jy, yi[ip]), dz = sub2(jz, zi[ip]);
                const float2 r2 = up2(fma2(dx, dx, fma2(dy, dy, mul2(dz, dz))));
                bits |= (r2.x <= rin2 ? 1u : 0u) << (2 * ip);
                bits |= (r2.y <= rin2 ? 1u : 0u) << (2 * ip + 1);
            }
            bits &= (unsigned)row[u].y & 0xffu;
            const unsigned keep = __ballot_sync(0xffffffffu, bits != 0u);
            if (bits) st.pl_row_in[base + out + __popc(keep & below)] = make_int2(row[u].x, (row[u].y & ~0xff) | (int)bits);
            out += __popc(keep);
        }
    }
    if (lane == 0) st.pl_count_in[ci] = out;
}

// Stages 1-7: the new slot order and the cluster boxes.  Everything but the
// pair kernel (bonded terms, PME, the learned descriptor) can run once this is
// done, concurrently with the pair search.
int launch_rebuild_slots(const DevState& st, bool from_input, cudaStream_t s) {
    const int TB = 256;
    const int nt = from_input ? st.n_atoms : st.n_slots;   // threads of the bin and scatter passes
    k_bin<<<(nt + TB - 1) / TB, TB, 0, s>>>(st, from_input ? 1 : 0);
    k_scan_columns<<<st.n_sys, 1024, 0, s>>>(st);
    k_scatter<<<(nt + TB - 1) / TB, TB, 0, s>>>(st, from_input ? 1 : 0);
    // keys for the next power of two of the column capacity (at most 8192: 64 KB)
    int m = 1;
    while (m < st.col_cap) m <<= 1;
    static std::atomic<unsigned long long> sort_attr{0ull};
    once_per_device(sort_attr, [] {
        cudaFuncSetAttribute(k_sort_columns, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             8192 * (int)sizeof(unsigned long long));
    });
    k_sort_columns<<<st.n_cols, 128, (size_t)m * sizeof(unsigned long long), s>>>(st, st.col_sys);
    k_gather_slots<<<(st.n_slots + TB - 1) / TB, TB, 0, s>>>(st, from_input ? 1 : 0);
    k_finish_slots<<<(st.n_slots + TB - 1) / TB, TB, 0, s>>>(st);
    k_bbox<<<(st.n_clusters + TB - 1) / TB, TB, 0, s>>>(st);
    return 7;
}

// Stage 8: the pair list of the current slots.
int launch_pairsearch(const DevState& st, float rlist, cudaStream_t s) {
    const int TP = PS_WARPS * 32;
    if (st.nb_split) {
        const long long threads = (long long)st.nb_warps * 32;
        k_pairsearch<true><<<(unsigned)((threads + TP - 1) / TP), TP, 0, s>>>(st, rlist);
        const long long tc = (long long)st.n_clusters * 32;
        k_pairsearch_concat<<<(unsigned)((tc + 255) / 256), 256, 0, s>>>(st);
        return 2;
    }
    const long long threads = (long long)st.n_clusters * 32;
    k_pairsearch<false><<<(unsigned)((threads + TP - 1) / TP), TP, 0, s>>>(st, rlist);
    return 1;
}

int launch_prune(const DevState& st, float rin, cudaStream_t s) {
    const long long threads = (long long)st.n_clusters * 32;
    k_prune_rows<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(st, rin * rin);
    return 1;
}

int launch_rebuild(const DevState& st, float rlist, bool from_input, cudaStream_t s) {
    return launch_rebuild_slots(st, from_input, s) + launch_pairsearch(st, rlist, s);
}

}  // namespace lima
