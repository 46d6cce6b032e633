// Row-partitioned BAIJ across ranks: the halo tables of BlockMatrix::set_halo
// (blockMatrix.hpp:317-348) and the device side of distributed_matvec
// (blockMatrix.hpp:351-437).  The exchange itself (the reference's
// MPI_Isend / MPI_Irecv) belongs to the caller's communicator -- NCCL through
// torch.distributed in the Python layer -- so this file provides the three
// device steps around it:
//   pack      send_buf[i] = x_owned[send_local[i]]            (before the exchange)
//   owned     y  = sum over owned-column blocks               (overlaps the exchange)
//   ghost     y += sum over ghost-column blocks of x_full     (after the exchange)
// with x_full = [x_owned | ghosts in recv order].  The sums follow the
// reference's MPI branch: y from zero, owned blocks in row order, then the
// ghost blocks, each block row component as acc = sum_c B[r][c] x_j[c] in c
// order -- so the result equals the reference's distributed_matvec bit for bit
// (which differs from the serial matvec in rounding: the two-phase order and
// no omp simd association).
#include "b2s_internal.cuh"

namespace b2s {

__global__ void k_ghost_pos(uint32_t n_ghost, const uint32_t* __restrict__ recv_global, uint32_t n_owned,
                            uint32_t* __restrict__ pos)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_ghost; k += gridDim.x * blockDim.x)
        pos[recv_global[k]] = n_owned + k;
}

// local column of every block; a column that is neither owned nor a listed
// ghost sets *bad (the reference would index past x_full)
__global__ void k_local_cols(uint32_t nnzb, const uint32_t* __restrict__ ci, uint32_t start, uint32_t n_owned,
                             const uint32_t* __restrict__ pos, uint32_t* __restrict__ lci, int* bad)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nnzb; p += gridDim.x * blockDim.x)
    {
        const uint32_t g = ci[p];
        uint32_t l;
        if (g >= start && g - start < n_owned)
            l = g - start;
        else
        {
            l = pos[g];
            if (l == 0xFFFFFFFFu)
            {
                atomicExch(bad, 1);
                l = 0;
            }
        }
        lci[p] = l;
    }
}

template <int BS>
__global__ void k_halo_pack(uint32_t n_send, const uint32_t* __restrict__ send_local, const double* __restrict__ x,
                            double* __restrict__ buf, const int* done)
{
    if (done && *done) return;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_send * BS; t += gridDim.x * blockDim.x)
        buf[t] = x[(size_t)send_local[t / BS] * BS + t % BS];
}

// one thread per block row component; GHOST = 0: y = owned part, 1: y += ghost part
template <int BS, int GHOST>
__global__ void k_dist_mv(uint32_t nbr, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ lci,
                          const double* __restrict__ v, uint32_t n_owned, const double* __restrict__ xf,
                          double* __restrict__ y, const int* done)
{
    if (done && *done) return;
    constexpr int BV = BS * BS;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nbr * BS; t += gridDim.x * blockDim.x)
    {
        const uint32_t bi = t / BS, r = t % BS;
        double yi = GHOST ? y[t] : 0.0;
        for (uint32_t p = rp[bi]; p < rp[bi + 1]; ++p)
        {
            const uint32_t j = lci[p];
            if ((j >= n_owned) != (GHOST != 0)) continue;
            const double* B = v + (size_t)p * BV + r * BS;
            const double* xj = xf + (size_t)j * BS;
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < BS; ++c) acc += B[c] * xj[c];
            yi += acc;
        }
        y[t] = yi;
    }
}

template <int GHOST>
static void dist_mv(b2s_ctx* ctx, const b2s_baij* A, const double* xf, double* y)
{
    const BaijDev& d = A->d;
    const HaloDev& h = A->halo;
    if (!d.nbr) return;
    const unsigned g = stream_grid(ctx, (uint64_t)d.nbr * d.bs);
    switch (d.bs)
    {
        case 1: B2S_LAUNCH(ctx, (k_dist_mv<1, GHOST>), g, kThreads, 0, d.nbr, d.rp.p, h.lci.p, d.v.p, h.n_owned, xf, y, nullptr); break;
        case 2: B2S_LAUNCH(ctx, (k_dist_mv<2, GHOST>), g, kThreads, 0, d.nbr, d.rp.p, h.lci.p, d.v.p, h.n_owned, xf, y, nullptr); break;
        case 3: B2S_LAUNCH(ctx, (k_dist_mv<3, GHOST>), g, kThreads, 0, d.nbr, d.rp.p, h.lci.p, d.v.p, h.n_owned, xf, y, nullptr); break;
        case 4: B2S_LAUNCH(ctx, (k_dist_mv<4, GHOST>), g, kThreads, 0, d.nbr, d.rp.p, h.lci.p, d.v.p, h.n_owned, xf, y, nullptr); break;
        default: fail(B2S_UNSUPPORTED, "block size must be 1..4");
    }
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_baij_set_halo(b2s_ctx* ctx, b2s_baij* A, int nrecv, const int* recv_procs, const int* recv_cnts,
                             const uint32_t* recv_global, int nsend, const int* send_procs, const int* send_cnts,
                             const uint32_t* send_local, uint32_t owned_global_start)
{
    if (!ctx || !A || nrecv < 0 || nsend < 0) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        const BaijDev& d = A->d;
        HaloDev h;
        h.n_owned = d.nbr;
        h.start = owned_global_start;
        need((uint64_t)owned_global_start + d.nbr <= d.nbc, B2S_INVALID_ARG,
             "set_halo: owned rows reach past the global block columns");
        uint64_t ng = 0, ns = 0;
        for (int k = 0; k < nrecv; ++k)
        {
            need(recv_cnts[k] >= 0, B2S_INVALID_ARG, "set_halo: negative receive count");
            ng += (uint64_t)recv_cnts[k];
            h.recv_procs.push_back(recv_procs[k]);
            h.recv_cnts.push_back(recv_cnts[k]);
        }
        for (int k = 0; k < nsend; ++k)
        {
            need(send_cnts[k] >= 0, B2S_INVALID_ARG, "set_halo: negative send count");
            ns += (uint64_t)send_cnts[k];
            h.send_procs.push_back(send_procs[k]);
            h.send_cnts.push_back(send_cnts[k]);
        }
        need(ng <= d.nbc && ns <= 0xFFFFFFFFull, B2S_INVALID_ARG, "set_halo: table sizes out of range");
        need(ng == 0 || recv_global, B2S_INVALID_ARG, "set_halo: null ghost list");
        need(ns == 0 || send_local, B2S_INVALID_ARG, "set_halo: null send list");
        for (uint64_t k = 0; k < ng; ++k)
        {
            const uint32_t g = recv_global[k];
            need(g < d.nbc && !(g >= owned_global_start && g - owned_global_start < d.nbr), B2S_INVALID_ARG,
                 "set_halo: a ghost column is out of range or owned by this rank");
        }
        for (uint64_t k = 0; k < ns; ++k)
            need(send_local[k] < d.nbr, B2S_INVALID_ARG, "set_halo: a send row is not an owned row");
        h.n_ghost = (uint32_t)ng;
        h.n_send = (uint32_t)ns;
        h.send_local = upload(ctx, send_local, ns);
        h.lci.alloc(d.nnzb ? d.nnzb : 1);
        DBuf<uint32_t> pos(d.nbc ? d.nbc : 1);
        DBuf<uint32_t> rg = upload(ctx, recv_global, ng);
        DBuf<int> bad(1);
        B2S_CUDA(cudaMemsetAsync(pos.p, 0xFF, pos.bytes(), ctx->stream));
        B2S_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
        if (ng) B2S_LAUNCH(ctx, k_ghost_pos, stream_grid(ctx, ng), kThreads, 0, (uint32_t)ng, rg.p, h.n_owned, pos.p);
        if (d.nnzb)
            B2S_LAUNCH(ctx, k_local_cols, stream_grid(ctx, d.nnzb), kThreads, 0, d.nnzb, d.ci.p, owned_global_start,
                       h.n_owned, pos.p, h.lci.p, bad.p);
        int hb = 0;
        d2h(ctx, &hb, bad.p, sizeof(int));
        sync(ctx);
        need(!hb, B2S_INVALID_ARG, "set_halo: a block column is neither owned nor in the ghost list");
        h.set = true;
        A->halo = std::move(h);
    });
}

b2s_status b2s_baij_halo_info(const b2s_baij* A, uint32_t* n_owned, uint32_t* n_ghost, uint32_t* n_send)
{
    if (!A || !A->halo.set) return B2S_INVALID_ARG;
    if (n_owned) *n_owned = A->halo.n_owned;
    if (n_ghost) *n_ghost = A->halo.n_ghost;
    if (n_send) *n_send = A->halo.n_send;
    return B2S_OK;
}

b2s_status b2s_baij_halo_pack_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x_owned, double* d_send_buf)
{
    if (!ctx || !A || !A->halo.set) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        const HaloDev& h = A->halo;
        if (!h.n_send) return;
        const unsigned g = stream_grid(ctx, (uint64_t)h.n_send * A->d.bs);
        switch (A->d.bs)
        {
            case 1: B2S_LAUNCH(ctx, k_halo_pack<1>, g, kThreads, 0, h.n_send, h.send_local.p, d_x_owned, d_send_buf, nullptr); break;
            case 2: B2S_LAUNCH(ctx, k_halo_pack<2>, g, kThreads, 0, h.n_send, h.send_local.p, d_x_owned, d_send_buf, nullptr); break;
            case 3: B2S_LAUNCH(ctx, k_halo_pack<3>, g, kThreads, 0, h.n_send, h.send_local.p, d_x_owned, d_send_buf, nullptr); break;
            case 4: B2S_LAUNCH(ctx, k_halo_pack<4>, g, kThreads, 0, h.n_send, h.send_local.p, d_x_owned, d_send_buf, nullptr); break;
        }
    });
}

b2s_status b2s_baij_dist_matvec_owned_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x_full, double* d_y)
{
    if (!ctx || !A || !A->halo.set) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { dist_mv<0>(ctx, A, d_x_full, d_y); });
}

b2s_status b2s_baij_dist_matvec_ghost_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x_full, double* d_y)
{
    if (!ctx || !A || !A->halo.set) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { dist_mv<1>(ctx, A, d_x_full, d_y); });
}

}  // extern "C"
