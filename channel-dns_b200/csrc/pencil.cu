// Pencil decomposition of one channel over several ranks: the reference's
// distributed path (INDEX_Serial = 0; Mesh's block tables,
// src/core/mesh.cpp:20-85; Transforms' transposes, src/fft/transforms.cpp:126-170
// and 304-404) re-planned for GPUs.
//
// Rank r holds the spectral state of one kx block [kx0_r, kx0_r + nkx_r)
// (every kz and Chebyshev mode) and, during a step, one slab [j0_r, j0_r + nj_r)
// of the NY2 + 1 fine-grid y points.  Every stage of the step is local to one
// of the two layouts:
//   kx block : curl, Chebyshev synthesis, Chebyshev analysis, column solve
//   y slab   : z synthesis, x stage (c2r, u x omega, r2c), z analysis
// so a step needs two all-to-all exchanges of the y-physical columns, between
// the Chebyshev and the z transforms: exchange 0 sends the six synthesised
// fields (u, omega) from kx blocks to y slabs, exchange 1 sends the three
// nonlinear-term fields back.  The reference runs one transpose per 3-D
// transform (nine per step) at the same point of each transform.
//
// The exchange itself is the caller's (NCCL all-to-all through
// torch.distributed, or device copies when the ranks share a process): this
// file packs each peer's chunk contiguously before it and unpacks after it.
// Packed chunk for peer q, element order [field][y][kz][kx]:
//   exchange 0 send / exchange 1 recv: y in q's slab,  kx in this rank's block
//   exchange 0 recv / exchange 1 send: y in this slab, kx in q's block
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "context.cuh"

namespace cdns {

constexpr int kMaxRanks = 64;

// The reference's block rule (src/core/mesh.cpp:28-40): n / P entries per
// rank, one more on each of the last n % P ranks, blocks in rank order.
static void split_blocks(int n, int P, int *begin, int *count) {
    const int base = n / P, extra = n % P;
    int b = 0;
    for (int r = 0; r < P; ++r) {
        count[r] = base + (r >= P - extra ? 1 : 0);
        begin[r] = b;
        b += count[r];
    }
}

int pencil_blocks(const cdns_mesh_desc &m, int ranks, int rank, int &kx0, int &nkx, int &j0, int &nj) {
    if (ranks < 1 || ranks > kMaxRanks) return fail(CDNS_ERR_ARG, "pencil ranks must be in 1..64");
    if (rank < 0 || rank >= ranks) return fail(CDNS_ERR_ARG, "invalid pencil rank");
    // src/core/mesh.cpp:22-24: no rank may receive an empty x, y or y2 block
    if (ranks > m.NXS + 1 || ranks > m.NY + 1 || ranks > m.NY2 + 1)
        return fail(CDNS_ERR_ARG, "pencil ranks exceed an x/y decomposition extent");
    int b[kMaxRanks], n[kMaxRanks];
    split_blocks(m.NXS + 1, ranks, b, n);
    kx0 = b[rank];
    nkx = n[rank];
    split_blocks(m.NY2 + 1, ranks, b, n);
    j0 = b[rank];
    nj = n[rank];
    return CDNS_OK;
}

namespace {

// One side of an exchange: the array [nf][ny_arr][nkz][nkx_arr] and, per
// peer q, its packed chunk at off[q]: rows[q] y rows from row0[q], width[q]
// kx columns from col0[q], element order [f][y][kz][kx].
struct PartMap {
    int nq, nf, nkz, ny_arr, nkx_arr;
    long long off[kMaxRanks + 1];
    int rows[kMaxRanks], row0[kMaxRanks], width[kMaxRanks], col0[kMaxRanks];
};

// Grid (chunk blocks, peers): block y = q copies chunk q.  32-bit index
// arithmetic inside a chunk (a chunk holds fewer than 2^30 values, checked
// when the map is built).
template <bool PACK>
__global__ void __launch_bounds__(256) k_part_copy(PartMap m, double2 *__restrict__ arr, double2 *__restrict__ packed) {
    const int q = blockIdx.y;
    const int n = (int)(m.off[q + 1] - m.off[q]);
    const int w = m.width[q], rows = m.rows[q];
    double2 *pk = packed + m.off[q];
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        int r = i;
        const int k = r % w;
        r /= w;
        const int kz = r % m.nkz;
        r /= m.nkz;
        const int j = r % rows;
        const int f = r / rows;
        const long long a = (((long long)f * m.ny_arr + m.row0[q] + j) * m.nkz + kz) * m.nkx_arr + m.col0[q] + k;
        if (PACK) pk[i] = arr[a];
        else arr[a] = pk[i];
    }
}

}  // namespace

struct PencilWork {
    int ranks = 1, rank = 0;
    int kx0[kMaxRanks], nkx[kMaxRanks], j0[kMaxRanks], nj[kMaxRanks];
    double2 *Fs = nullptr, *Gs = nullptr, *Hs = nullptr;   // y-slab stage buffers
    double2 *buf[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [exchange][send, recv]
    long long count[2][2] = {{0, 0}, {0, 0}};                        // complex values
    // exchange 0: block side packs (send), slab side unpacks (recv);
    // exchange 1: slab side packs (send), block side unpacks (recv)
    PartMap block[2], slab[2];
    int next_stage = 0, iteration = 0;
    long long chunk_max[2][2] = {{0, 0}, {0, 0}};
    // fused exchange (cdns_pencil_set_peers): per global kx, the owning rank's
    // column pointer and row stride; the z transforms then read and write
    // every rank's column buffer directly and the exchange buffers are idle
    double2 **col = nullptr;
    int *width = nullptr;
    bool peers = false;
    std::vector<void *> opened;   // peers' column buffers mapped from CUDA IPC handles
};

void pencil_release(PencilWork *w) {
    if (!w) return;
    for (void *p : w->opened) cudaIpcCloseMemHandle(p);
    delete w;
}

namespace {

// The y-slab view of a rank: every kx, the rank's nj y points.
Dims slab_dims(const cdns_ctx *c) {
    const PencilWork &w = *c->pen;
    Dims ds = c->d;
    ds.kx0 = 0;
    ds.zc = -1;
    ds.nkx = ds.NXS + 1;
    ds.ncol = ds.nkx * ds.nkz;
    ds.fcol = ds.ncol;
    ds.ny2 = w.nj[w.rank];
    ds.Ns = (long long)ds.nkz * ds.ncy * ds.nkx;
    return ds;
}

int build_map(PartMap &m, int nf, int nkz, int ny_arr, int nkx_arr, int P, const int *rows, const int *row0,
              const int *width, const int *col0, long long &max_chunk) {
    m.nq = P;
    m.nf = nf;
    m.nkz = nkz;
    m.ny_arr = ny_arr;
    m.nkx_arr = nkx_arr;
    m.off[0] = 0;
    max_chunk = 0;
    for (int q = 0; q < P; ++q) {
        if (row0[q] < 0 || rows[q] < 1 || row0[q] + rows[q] > ny_arr || col0[q] < 0 || width[q] < 1 ||
            col0[q] + width[q] > nkx_arr)
            return fail(CDNS_ERR_ARG, "pencil exchange map out of the array");
        m.rows[q] = rows[q];
        m.row0[q] = row0[q];
        m.width[q] = width[q];
        m.col0[q] = col0[q];
        const long long n = (long long)nf * rows[q] * nkz * width[q];
        // int index arithmetic in k_part_copy, grid stride included
        if (n >= (1LL << 30)) return fail(CDNS_ERR_ARG, "pencil exchange chunk exceeds 2^30 values");
        m.off[q + 1] = m.off[q] + n;
        max_chunk = std::max(max_chunk, n);
    }
    return CDNS_OK;
}

int part_copy(const PartMap &m, long long max_chunk, bool pack, double2 *arr, double2 *packed, cudaStream_t s) {
    if (max_chunk == 0) return CDNS_OK;
    const long long blocks = std::min<long long>((max_chunk + 255) / 256, 1184);
    dim3 grid((unsigned)blocks, (unsigned)m.nq);
    if (pack) k_part_copy<true><<<grid, 256, 0, s>>>(m, arr, packed);
    else k_part_copy<false><<<grid, 256, 0, s>>>(m, arr, packed);
    CK(cudaGetLastError());
    return CDNS_OK;
}

}  // namespace

int pencil_init(cdns_ctx *c, int ranks, int rank) {
    PencilWork *w = new (std::nothrow) PencilWork();
    if (!w) return fail(CDNS_ERR_NOMEM, "host allocation failed");
    c->pen = w;
    w->ranks = ranks;
    w->rank = rank;
    for (int q = 0; q < ranks; ++q) {
        int r = pencil_blocks(c->mesh, ranks, q, w->kx0[q], w->nkx[q], w->j0[q], w->nj[q]);
        if (r) return r;
    }
    const Dims &d = c->d;
    const Dims ds = slab_dims(c);
    const int me = rank, nkz = d.nkz, ny2 = d.ny2, nkxg = ds.nkx;
    const int njme = w->nj[me], nkxme = w->nkx[me];
    int zeros[kMaxRanks], njme_v[kMaxRanks], nkxme_v[kMaxRanks];
    for (int q = 0; q < ranks; ++q) {
        zeros[q] = 0;
        njme_v[q] = njme;
        nkxme_v[q] = nkxme;
    }
    int r;
    // block side [f][NY2+1][kz][kx block]: peer q's chunk is q's y slab
    // slab side [f][nj][kz][every kx]: peer q's chunk is q's kx block
    if ((r = build_map(w->block[0], 6, nkz, ny2, nkxme, ranks, w->nj, w->j0, nkxme_v, zeros, w->chunk_max[0][0])) ||
        (r = build_map(w->slab[0], 6, nkz, njme, nkxg, ranks, njme_v, zeros, w->nkx, w->kx0, w->chunk_max[0][1])) ||
        (r = build_map(w->slab[1], 3, nkz, njme, nkxg, ranks, njme_v, zeros, w->nkx, w->kx0, w->chunk_max[1][0])) ||
        (r = build_map(w->block[1], 3, nkz, ny2, nkxme, ranks, w->nj, w->j0, nkxme_v, zeros, w->chunk_max[1][1])))
        return r;
    w->count[0][0] = w->block[0].off[ranks];
    w->count[0][1] = w->slab[0].off[ranks];
    w->count[1][0] = w->slab[1].off[ranks];
    w->count[1][1] = w->block[1].off[ranks];
    const size_t zslab = (size_t)njme * d.NZ2 * nkxg;
    if ((r = c->alloc(w->Fs, 6 * (size_t)njme * nkz * nkxg)) || (r = c->alloc(w->Gs, 6 * zslab)) ||
        (r = c->alloc(w->Hs, 3 * zslab)))
        return r;
    for (int e = 0; e < 2; ++e)
        for (int k = 0; k < 2; ++k)
            if ((r = c->alloc(w->buf[e][k], (size_t)w->count[e][k]))) return r;
    if ((r = c->alloc(w->col, (size_t)nkxg)) || (r = c->alloc(w->width, (size_t)nkxg))) return r;
    cudaError_t err = configure_transform_kernels(ds);
    if (err != cudaSuccess) return fail(CDNS_ERR_CUDA, cudaGetErrorString(err));
    return CDNS_OK;
}

}  // namespace cdns

using namespace cdns;

extern "C" {

int cdns_pencil_layout(const cdns_mesh_desc *m, int ranks, int *table) {
    if (!m || !table) return fail(CDNS_ERR_ARG, "null argument");
    for (int q = 0; q < ranks; ++q) {
        int r = pencil_blocks(*m, ranks, q, table[4 * q], table[4 * q + 1], table[4 * q + 2], table[4 * q + 3]);
        if (r) return r;
    }
    if (ranks < 1) return fail(CDNS_ERR_ARG, "pencil ranks must be in 1..64");
    return CDNS_OK;
}

int cdns_pencil_counts(const cdns_mesh_desc *m, int ranks, int rank, int exchange, long long *send,
                       long long *recv) {
    if (!m || !send || !recv) return fail(CDNS_ERR_ARG, "null argument");
    if (exchange != 0 && exchange != 1) return fail(CDNS_ERR_ARG, "exchange must be 0 or 1");
    int kx0, nkxme, j0, njme;
    int r = pencil_blocks(*m, ranks, rank, kx0, nkxme, j0, njme);
    if (r) return r;
    const long long nkz = 2LL * m->NZS + 1;
    for (int q = 0; q < ranks; ++q) {
        int qk0, qnkx, qj0, qnj;
        if ((r = pencil_blocks(*m, ranks, q, qk0, qnkx, qj0, qnj))) return r;
        // doubles: block-side chunk (q's slab x my block), slab-side chunk (my slab x q's block)
        const long long block = 2 * (long long)qnj * nkz * nkxme, slab = 2 * (long long)njme * nkz * qnkx;
        send[q] = exchange == 0 ? 6 * block : 3 * slab;
        recv[q] = exchange == 0 ? 6 * slab : 3 * block;
    }
    return CDNS_OK;
}

int cdns_pencil_buffer(cdns_ctx *c, int exchange, int recv, void **ptr, long long *doubles) {
    if (!c || !ptr || !doubles) return fail(CDNS_ERR_ARG, "null argument");
    if (!c->pen) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    if ((exchange != 0 && exchange != 1) || (recv != 0 && recv != 1))
        return fail(CDNS_ERR_ARG, "exchange and recv must be 0 or 1");
    *ptr = c->pen->buf[exchange][recv];
    *doubles = 2 * c->pen->count[exchange][recv];
    return CDNS_OK;
}

int cdns_pencil_columns(cdns_ctx *c, void **ptr, long long *doubles) {
    if (!c || !ptr || !doubles) return fail(CDNS_ERR_ARG, "null argument");
    if (!c->pen) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    *ptr = c->F;
    *doubles = 2LL * 6 * c->d.ny2 * c->d.ncol;
    return CDNS_OK;
}

int cdns_pencil_ipc_handle(cdns_ctx *c, void *handle) {
    if (!c || !handle) return fail(CDNS_ERR_ARG, "null argument");
    if (!c->pen) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    static_assert(sizeof(cudaIpcMemHandle_t) == CDNS_IPC_HANDLE_BYTES, "IPC handle size");
    DeviceGuard guard(c->device);
    cudaIpcMemHandle_t h;
    CK(cudaIpcGetMemHandle(&h, c->F));
    std::memcpy(handle, &h, sizeof h);
    return CDNS_OK;
}

int cdns_pencil_close_peers(cdns_ctx *c) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (!c->pen) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    if (c->pen->next_stage != 0) return fail(CDNS_ERR_STATE, "cdns_pencil_close_peers inside a step");
    DeviceGuard guard(c->device);
    CK(cudaStreamSynchronize(c->stream));   // no stage of this rank still reads a peer's buffer
    c->pen->peers = false;
    for (void *p : c->pen->opened) CK(cudaIpcCloseMemHandle(p));
    c->pen->opened.clear();
    return CDNS_OK;
}

int cdns_pencil_open_peer(cdns_ctx *c, const void *handle, void **ptr) {
    if (!c || !handle || !ptr) return fail(CDNS_ERR_ARG, "null argument");
    if (!c->pen) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    DeviceGuard guard(c->device);
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof h);
    void *p = nullptr;
    CK(cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess));
    c->pen->opened.push_back(p);
    *ptr = p;
    return CDNS_OK;
}

// A peer's column buffer must be device memory that this context's device
// can reach (its own, or a peer device with access enabled here, which this
// call enables), and it must hold `bytes` from `p` on (checked with the
// driver's address-range query where the driver offers it).  Anything else
// is refused before a kernel could fault on it.
static int check_peer_columns(cdns_ctx *c, const void *p, unsigned long long bytes) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || a.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return fail(CDNS_ERR_ARG, "peer column buffer is not device memory");
    }
    if (a.device != c->device) {
        int can = 0;
        CK(cudaDeviceCanAccessPeer(&can, c->device, a.device));
        if (!can) return fail(CDNS_ERR_ARG, "peer column buffer is on a device this device cannot access");
        const cudaError_t e = cudaDeviceEnablePeerAccess(a.device, 0);
        if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
        else if (e != cudaSuccess) return fail(CDNS_ERR_CUDA, cudaGetErrorString(e));
    }
    using RangeFn = int (*)(unsigned long long *, size_t *, unsigned long long);
    static RangeFn range = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        cudaGetLastError();
        return reinterpret_cast<RangeFn>(fn);
    }();
    if (range) {
        unsigned long long base = 0;
        size_t size = 0;
        if (range(&base, &size, reinterpret_cast<unsigned long long>(p)) == 0 &&
            reinterpret_cast<unsigned long long>(p) + bytes > base + size)
            return fail(CDNS_ERR_ARG, "peer column buffer is smaller than the rank's columns");
    }
    return CDNS_OK;
}

int cdns_pencil_set_peers(cdns_ctx *c, void *const *columns) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    PencilWork *w = c->pen;
    if (!w) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    if (w->next_stage != 0) return fail(CDNS_ERR_STATE, "cdns_pencil_set_peers inside a step");
    DeviceGuard guard(c->device);
    if (!columns) {
        w->peers = false;
        return CDNS_OK;
    }
    const Dims ds = slab_dims(c);
    if (!register_forms(ds)) return fail(CDNS_ERR_ARG, "the fused exchange needs NZ2 and NX2 with a register split");
    const int nkxg = c->d.NXS + 1;
    std::vector<double2 *> col(nkxg);
    std::vector<int> width(nkxg);
    for (int q = 0; q < w->ranks; ++q)
        if (!columns[q]) return fail(CDNS_ERR_ARG, "null peer column buffer");
    if (columns[w->rank] != static_cast<void *>(c->F))
        return fail(CDNS_ERR_ARG, "this rank's entry must be its own column buffer");
    for (int q = 0; q < w->ranks; ++q) {
        if (int r = check_peer_columns(c, columns[q], 16ull * 6 * c->d.ny2 * c->d.nkz * w->nkx[q])) return r;
        for (int k = 0; k < w->nkx[q]; ++k) {
            col[w->kx0[q] + k] = static_cast<double2 *>(columns[q]) + k;
            width[w->kx0[q] + k] = w->nkx[q];
        }
    }
    CK(cudaMemcpyAsync(w->col, col.data(), sizeof(double2 *) * nkxg, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(w->width, width.data(), sizeof(int) * nkxg, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    w->peers = true;
    return CDNS_OK;
}

int cdns_pencil_stage(cdns_ctx *c, int iteration, int stage) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    PencilWork *w = c->pen;
    if (!w) return fail(CDNS_ERR_STATE, "not a pencil rank context");
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "cdns_pencil_stage before cdns_set_velocity");
    if (iteration < 1) return fail(CDNS_ERR_ARG, "iteration must be >= 1");
    if (stage != w->next_stage || (stage > 0 && iteration != w->iteration))
        return fail(CDNS_ERR_STATE, "pencil stages run 0, 1, 2 for one iteration");
    DeviceGuard guard(c->device);
    cudaStream_t s = c->stream;
    const Dims &d = c->d;
    const int k = c->cur;
    double a0, a1, b0, b1, g;
    step_coefficients(iteration, c->DT, c->pp.Re, a0, a1, b0, b1, g);
    int r = CDNS_OK;
    if (stage == 0) {
        // EqSolvePV::setup at it = 1, 2 (src/sim/simulation.cpp:176-177)
        if ((r = do_setup(c, g))) return r;
        launch_curl(d, c->t, c->U[k], c->om, c->bw, c->pp.Re, s);
        launch_ysynth(d, c->t, c->U[k], c->om, 3, 6, c->F, s);
        if (!w->peers) r = part_copy(w->block[0], w->chunk_max[0][0], true, c->F, w->buf[0][0], s);
    } else if (stage == 1) {
        const Dims ds = slab_dims(c);
        if (w->peers) {
            const PeerCols pc{w->col, w->width, d.ny2, w->j0[w->rank]};
            if (!launch_z_backward_peers(ds, c->t.root_z, pc, w->Gs, s))
                return fail(CDNS_ERR_ARG, "the fused exchange needs NZ2 with a register split");
            launch_x_cross(ds, c->px, c->t.root_x, w->Gs, w->Hs, s);
            launch_z_forward_peers(ds, c->t.root_z, w->Hs, pc, s);
        } else {
            if ((r = part_copy(w->slab[0], w->chunk_max[0][1], false, w->Fs, w->buf[0][1], s))) return r;
            launch_z_backward(ds, c->pz, c->t.root_z, w->Fs, w->Gs, 6, s);
            launch_x_cross(ds, c->px, c->t.root_x, w->Gs, w->Hs, s);
            launch_z_forward(ds, c->pz, c->t.root_z, w->Hs, w->Fs, 3, s);
            r = part_copy(w->slab[1], w->chunk_max[1][0], true, w->Fs, w->buf[1][0], s);
        }
    } else if (stage == 2) {
        if (!w->peers && (r = part_copy(w->block[1], w->chunk_max[1][1], false, c->F, w->buf[1][1], s)))
            return r;
        launch_yanalysis(d, c->t, c->F, c->Nb[k], 3, s);
        enqueue_solve(c, a0, a1, b0, b1, g);
        c->cur = 1 - k;
    } else {
        return fail(CDNS_ERR_ARG, "stage must be 0, 1 or 2");
    }
    if (r) return r;
    CK(cudaGetLastError());
    w->iteration = iteration;
    w->next_stage = (stage + 1) % 3;
    return CDNS_OK;
}

}  // extern "C"
