// Decomposed HPCG problem: one rank's sub-brick on one GPU, its halo plan on
// every MG level, the halo exchange and the distributed CG (FP64 ELL path).
//
// A rank's local matrix is the single-rank matrix of its brick (same JPL
// colouring, permutation and column order: the colouring and the column sort
// only look at local columns, src/MultiColoring.cpp:193, src/Permute.cpp:
// 109-121) with the external entries appended after the local ones in each
// row's ELL slots, as the reference's key sort leaves them.  The operators
// follow the reference's multi-rank sequence (src/ComputeSPMV.cpp:226-278,
// src/ComputeSYMGS.cpp:369-404, src/ComputeRestriction.cpp:199-237,
// src/ComputeMG.cpp:64-102, src/CG.cpp:104-200, src/ComputeDotProduct.cpp:
// 189-238): gather the send buffer, start the exchange, run the interior
// kernel (local columns), complete the exchange, run the halo kernel.
//
// Two transports carry the exchange and the cross-rank sums:
//  * NCCL (one process per GPU): send/recv of the packed faces into the
//    receiving rank's own memory on a communication stream that overlaps the
//    interior kernel, and an 8-byte allreduce per dot product, all
//    stream-ordered (no host round trip inside an iteration);
//  * a group of every rank driven from one process on one device: the
//    exchange is a device-to-device copy per neighbour and the sums a kernel
//    over the ranks' scalars, all launched in order on one stream (no kernel
//    ever waits for another).
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>

#include <nccl.h>

#include "../csrc/halo.cuh"
#include "dist.hpp"
#include "hpcg_b200.h"
#include "internal.hpp"
#include "problem.hpp"

using namespace hpcg_b200;

namespace hpcg_b200 {
namespace {

// ------------------------------------------------------------ NCCL, at run time
// Loaded with dlopen so that the library loads (and its host logic runs)
// where NCCL is absent; in a process that already mapped libnccl.so.2 (e.g.
// through torch) the same copy is used.
struct NcclApi
{
    bool tried = false, ok = false;
    std::string why;
    ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
    ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

NcclApi& nccl()
{
    static NcclApi a;
    if(a.tried) return a;
    a.tried = true;
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if(!h)
    {
        const char* e = dlerror();
        a.why = e ? e : "dlopen failed";
        return a;
    }
    bool ok = true;
    auto get = [&](auto& fn, const char* name) {
        fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
        if(!fn) ok = false;
    };
    get(a.GetUniqueId, "ncclGetUniqueId");
    get(a.CommInitRank, "ncclCommInitRank");
    get(a.CommDestroy, "ncclCommDestroy");
    get(a.CommAbort, "ncclCommAbort");
    get(a.Send, "ncclSend");
    get(a.Recv, "ncclRecv");
    get(a.AllReduce, "ncclAllReduce");
    get(a.GroupStart, "ncclGroupStart");
    get(a.GroupEnd, "ncclGroupEnd");
    get(a.GetErrorString, "ncclGetErrorString");
    a.ok = ok;
    if(!ok) a.why = "libnccl.so.2 lacks a needed symbol";
    return a;
}

void check_nccl(ncclResult_t r, const char* what)
{
    if(r == ncclSuccess) return;
    char buf[256];
    snprintf(buf, sizeof(buf), "NCCL error %d (%s) in %s", (int)r, nccl().GetErrorString(r), what);
    throw Error(HPCGB200_ERR_COMM, buf);
}

// Steady CG iterations as one CUDA graph launch each (HPCGB200_DIST_GRAPH=0:
// direct launches).
bool dist_graphs()
{
    const char* e = std::getenv("HPCGB200_DIST_GRAPH");
    return !e || std::atoi(e) != 0;
}

double dist_timeout_s()
{
    const char* e = std::getenv("HPCGB200_DIST_TIMEOUT_S");
    const double v = e ? std::atof(e) : 0.0;
    return v > 0.0 ? v : 600.0;
}

// ------------------------------------------------------------ per-level data
struct DistLevel
{
    SparseMatrix* A = nullptr;
    DistGeom g;
    HaloPlan plan;
    int m = 0, ncols = 0, nsend = 0, nh = 0, hw = 0;
    long long nnz = 0;           // nonzeros of this rank's rows, external ones included
    int* send_perm = nullptr;    // permuted local row of each send-buffer entry
    double* send_buf = nullptr;
    int* prow = nullptr;         // permuted row of each halo row
    int* hcol = nullptr;         // column-major external columns (hw x nh, -1 padded)
    double* hval = nullptr;
    int* pc = nullptr;           // coarse permuted row a halo row injects into (-1: none)
    double* xv = nullptr;        // levels >= 1: the level's x (local rows + external tail)
    double* rv = nullptr;        // levels >= 1: the level's right-hand side
};

}  // namespace
}  // namespace hpcg_b200

struct hpcgb200_halo_plan
{
    hpcg_b200::DistGeom g;
    hpcg_b200::HaloPlan plan;
};

struct hpcgb200_dist
{
    hpcgb200_problem* local = nullptr;  // the rank's brick as a single-rank problem (levels, colouring, ELL)
    std::vector<hpcg_b200::DistLevel> L;
    int size = 1, rank = 0;
    double *x = nullptr, *p = nullptr, *z = nullptr;  // level 0, local rows + external tail
    double *r = nullptr, *Ap = nullptr;
    double* b_gen = nullptr;                          // generated b (27 - nonzeros per row), permuted
    double* sc = nullptr;                             // DistSlot scalars
    double* h_sc = nullptr;                           // pinned mirror
    int* d_status = nullptr;
    ncclComm_t comm = nullptr;
    cudaStream_t comm_stream = nullptr;
    cudaEvent_t ev_packed = nullptr, ev_recv = nullptr, ev_sync = nullptr;
    unsigned long long serial = 0;                    // process-unique id (graph cache keys)
    // cached CUDA graph of one steady CG iteration of a group whose first rank
    // is this one: the group's serials and the preconditioner flag as its key
    std::vector<unsigned long long> graph_key;
    bool graph_precond = false;
    cudaGraphExec_t graph_exec = nullptr;
};

namespace hpcg_b200 {
namespace {

// ------------------------------------------------------------ groups
struct Group
{
    std::vector<hpcgb200_dist*> R;
    std::vector<int> pos;  // rank id -> index in R (emulated groups)
    bool use_nccl = false;
    cudaStream_t s = nullptr;
    int nlevels = 0;
};

Group make_group(hpcgb200_dist* const* ranks, int n)
{
    if(!ranks || n < 1) throw Error(HPCGB200_ERR_ARG, "empty rank group");
    Group G;
    G.s = rt().stream;
    G.R.assign(ranks, ranks + n);
    for(auto* d : G.R)
        if(!d) throw Error(HPCGB200_ERR_ARG, "null rank in group");
    const int size = G.R[0]->size;
    G.nlevels = (int)G.R[0]->L.size();
    if(n == 1)
    {
        // a rank with a communicator always goes through NCCL (for one rank:
        // no exchange, a one-rank allreduce)
        G.use_nccl = G.R[0]->comm != nullptr;
        if(size > 1 && !G.use_nccl)
            throw Error(HPCGB200_ERR_ARG, "a rank of a decomposed problem solves alone only with a communicator "
                                          "(hpcgb200_dist_attach_nccl), or drive all ranks as one group");
        return G;
    }
    if(n != size || n > hb::kMaxGroup)
        throw Error(HPCGB200_ERR_ARG, "a group holds every rank of one decomposition (at most 64)");
    G.pos.assign(size, -1);
    const DistGeom& g0 = G.R[0]->L[0].g;
    for(int i = 0; i < n; ++i)
    {
        const DistGeom& g = G.R[i]->L[0].g;
        if(G.R[i]->size != size || (int)G.R[i]->L.size() != G.nlevels || g.nx != g0.nx || g.ny != g0.ny ||
           g.nz != g0.nz || g.npx != g0.npx || g.npy != g0.npy || g.npz != g0.npz)
            throw Error(HPCGB200_ERR_ARG, "group ranks come from different decompositions");
        if(G.pos[G.R[i]->rank] >= 0)
            throw Error(HPCGB200_ERR_ARG, "rank " + std::to_string(G.R[i]->rank) + " twice in the group");
        G.pos[G.R[i]->rank] = i;
    }
    return G;
}

template <typename F>
void each(Group& G, F&& f)
{
    for(size_t i = 0; i < G.R.size(); ++i) check(f(G.R[i], (int)i));
}

// Send buffers are packed (on G.s); the external tails of xs[i] receive.
void exchange_begin(Group& G, int l, const std::vector<double*>& xs)
{
    TraceRange trace("hpcg:ExchangeHalo");
    if(G.use_nccl)
    {
        hpcgb200_dist* d = G.R[0];
        const DistLevel& Lv = d->L[l];
        const HaloPlan& P = Lv.plan;
        if(P.nbr_rank.empty()) return;
        NcclApi& N = nccl();
        HB_HOST_CUDA(cudaEventRecord(d->ev_packed, G.s));
        HB_HOST_CUDA(cudaStreamWaitEvent(d->comm_stream, d->ev_packed, 0));
        check_nccl(N.GroupStart(), "ncclGroupStart");
        for(size_t j = 0; j < P.nbr_rank.size(); ++j)
        {
            check_nccl(N.Recv(xs[0] + Lv.m + P.recv_off[j], (size_t)P.recv_len[j], ncclFloat64, P.nbr_rank[j], d->comm,
                              d->comm_stream),
                       "ncclRecv");
            check_nccl(N.Send(Lv.send_buf + P.send_off[j], (size_t)P.send_len[j], ncclFloat64, P.nbr_rank[j], d->comm,
                              d->comm_stream),
                       "ncclSend");
        }
        check_nccl(N.GroupEnd(), "ncclGroupEnd");
        HB_HOST_CUDA(cudaEventRecord(d->ev_recv, d->comm_stream));
        return;
    }
    if(G.R.size() == 1) return;
    for(size_t i = 0; i < G.R.size(); ++i)
    {
        hpcgb200_dist* d = G.R[i];
        const DistLevel& Lv = d->L[l];
        const HaloPlan& P = Lv.plan;
        for(size_t j = 0; j < P.nbr_rank.size(); ++j)
        {
            const hpcgb200_dist* src = G.R[G.pos[P.nbr_rank[j]]];
            const DistLevel& Ls = src->L[l];
            const HaloPlan& Q = Ls.plan;
            size_t k = 0;
            while(k < Q.nbr_rank.size() && Q.nbr_rank[k] != d->rank) ++k;
            if(k == Q.nbr_rank.size() || Q.send_len[k] != P.recv_len[j])
                throw Error(HPCGB200_ERR_ARG, "halo plans of ranks " + std::to_string(d->rank) + " and " +
                                                  std::to_string(src->rank) + " disagree");
            HB_HOST_CUDA(cudaMemcpyAsync(xs[i] + Lv.m + P.recv_off[j], Ls.send_buf + Q.send_off[k],
                                         sizeof(double) * P.recv_len[j], cudaMemcpyDeviceToDevice, G.s));
        }
    }
}

void exchange_end(Group& G, int l)
{
    if(!G.use_nccl) return;
    hpcgb200_dist* d = G.R[0];
    if(d->L[l].plan.nbr_rank.empty()) return;
    HB_HOST_CUDA(cudaStreamWaitEvent(G.s, d->ev_recv, 0));
}

void pack(Group& G, int l, const std::vector<double*>& xs)
{
    each(G, [&](hpcgb200_dist* d, int i) {
        const DistLevel& Lv = d->L[l];
        return hb::launch_halo_pack(Lv.nsend, Lv.send_perm, xs[i], Lv.send_buf, G.s);
    });
}

// Sum of slot `k` of every rank's scalars, left in every rank's slot.
void allreduce(Group& G, int k)
{
    TraceRange trace("hpcg:Allreduce");
    if(G.use_nccl)
    {
        hpcgb200_dist* d = G.R[0];
        check_nccl(nccl().AllReduce(d->sc + k, d->sc + k, 1, ncclFloat64, ncclSum, d->comm, G.s), "ncclAllReduce");
        return;
    }
    if(G.R.size() == 1) return;
    hb::SlotPtrs P{};
    for(size_t i = 0; i < G.R.size(); ++i) P.p[i] = G.R[i]->sc + k;
    check(hb::launch_group_sum((int)G.R.size(), P, G.s));
}

// Waits for G.s.  With NCCL the wait is bounded: a peer that stopped leaves
// the collectives pending, and after HPCGB200_DIST_TIMEOUT_S seconds (600 by
// default) the communicator is aborted and the call fails.
void wait_stream(Group& G)
{
    if(!G.use_nccl)
    {
        HB_HOST_CUDA(cudaStreamSynchronize(G.s));
        return;
    }
    hpcgb200_dist* d = G.R[0];
    HB_HOST_CUDA(cudaEventRecord(d->ev_sync, G.s));
    const auto t0 = std::chrono::steady_clock::now();
    const double limit = dist_timeout_s();
    for(long long n = 0;; ++n)
    {
        const cudaError_t e = cudaEventQuery(d->ev_sync);
        if(e == cudaSuccess) return;
        if(e != cudaErrorNotReady) check_cuda(e, "cudaEventQuery");
        if((n & 1023) == 1023)
        {
            if(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit)
            {
                nccl().CommAbort(d->comm);
                d->comm = nullptr;
                throw Error(HPCGB200_ERR_COMM, "decomposed solve: no progress for " + std::to_string(limit) +
                                                   " s (a peer stopped?); communicator aborted");
            }
            std::this_thread::yield();
        }
    }
}

double read_slot(Group& G, int k)
{
    hpcgb200_dist* d = G.R[0];
    HB_HOST_CUDA(cudaMemcpyAsync(d->h_sc + k, d->sc + k, sizeof(double), cudaMemcpyDeviceToHost, G.s));
    wait_stream(G);
    return d->h_sc[k];
}

// ------------------------------------------------------------ operators
void spmv(Group& G, int l, const std::vector<double*>& xs, const std::vector<double*>& ys)
{
    pack(G, l, xs);
    exchange_begin(G, l, xs);
    each(G, [&](hpcgb200_dist* d, int i) {
        const SparseMatrix& A = *d->L[l].A;
        return hb::launch_spmv(A.localNumberOfRows, opt(A)->cc, A.ell_col_ind, A.ell_val, xs[i], ys[i], G.s);
    });
    exchange_end(G, l);
    each(G, [&](hpcgb200_dist* d, int i) {
        const DistLevel& Lv = d->L[l];
        return hb::launch_halo_spmv(Lv.nh, Lv.hw, Lv.prow, Lv.hcol, Lv.hval, xs[i], ys[i], G.s);
    });
}

void symgs(Group& G, int l, const std::vector<double*>& rs, const std::vector<double*>& xs)
{
    pack(G, l, xs);
    exchange_begin(G, l, xs);
    each(G, [&](hpcgb200_dist* d, int i) {  // colour 0 on the local columns
        const SparseMatrix& A = *d->L[l].A;
        return hb::launch_sweep_color(A.localNumberOfRows, A.localNumberOfRows, A.sizes[0], A.offsets[0],
                                      A.ell_col_ind, A.ell_val, A.inv_diag, rs[i], xs[i], G.s);
    });
    exchange_end(G, l);
    each(G, [&](hpcgb200_dist* d, int i) {
        const DistLevel& Lv = d->L[l];
        const SparseMatrix& A = *Lv.A;
        check(hb::launch_halo_symgs0(Lv.nh, Lv.hw, Lv.prow, Lv.hcol, Lv.hval, A.inv_diag, A.sizes[0], xs[i], G.s));
        const int m = A.localNumberOfRows;
        for(int c = 1; c < A.nblocks; ++c)
            check(hb::launch_sweep_color(m, Lv.ncols, A.sizes[c], A.offsets[c], A.ell_col_ind, A.ell_val, A.inv_diag,
                                         rs[i], xs[i], G.s));
        for(int c = A.ublocks; c >= 0; --c)
            check(hb::launch_sweep_color(m, Lv.ncols, A.sizes[c], A.offsets[c], A.ell_col_ind, A.ell_val, A.inv_diag,
                                         rs[i], xs[i], G.s));
        return 0;
    });
}

void symgs_zero(Group& G, int l, const std::vector<double*>& rs, const std::vector<double*>& xs)
{
    each(G, [&](hpcgb200_dist* d, int i) {
        const SparseMatrix& A = *d->L[l].A;
        return hb::launch_symgs_zero(A.localNumberOfRows, A.nblocks, A.ublocks, A.sizes, A.offsets, A.ell_col_ind,
                                     A.ell_val, A.diag_idx, opt(A)->diag, A.inv_diag, rs[i], xs[i], G.s, {}, zg_of(A));
    });
}

void restrict_fused(Group& G, int l, const std::vector<double*>& rfs, const std::vector<double*>& xfs,
                    const std::vector<double*>& rcs)
{
    pack(G, l, xfs);
    exchange_begin(G, l, xfs);
    each(G, [&](hpcgb200_dist* d, int i) {
        const SparseMatrix& A = *d->L[l].A;
        const MGOpt* mo = mgopt(A);
        return hb::launch_restrict(A.Ac->localNumberOfRows, mo->inj_f, mo->inj_c, A.localNumberOfRows, A.ell_col_ind,
                                   A.ell_val, rfs[i], xfs[i], rcs[i], G.s);
    });
    exchange_end(G, l);
    each(G, [&](hpcgb200_dist* d, int i) {
        const DistLevel& Lv = d->L[l];
        return hb::launch_halo_restrict(Lv.nh, Lv.hw, Lv.pc, Lv.hcol, Lv.hval, xfs[i], rcs[i], G.s);
    });
}

void prolong(Group& G, int l, const std::vector<double*>& xcs, const std::vector<double*>& xfs)
{
    each(G, [&](hpcgb200_dist* d, int i) {
        const SparseMatrix& A = *d->L[l].A;
        const MGOpt* mo = mgopt(A);
        return hb::launch_prolong(A.Ac->localNumberOfRows, mo->inj_f, mo->inj_c, xcs[i], xfs[i], G.s);
    });
}

std::vector<double*> level_vec(Group& G, int l, bool rhs)
{
    std::vector<double*> v;
    for(auto* d : G.R) v.push_back(rhs ? d->L[l].rv : d->L[l].xv);
    return v;
}

// src/ComputeMG.cpp:64-102 on every rank.
void mg(Group& G, int l, const std::vector<double*>& rs, const std::vector<double*>& xs)
{
    symgs_zero(G, l, rs, xs);
    if(l + 1 >= G.nlevels) return;
    const auto rc = level_vec(G, l + 1, true), xc = level_vec(G, l + 1, false);
    restrict_fused(G, l, rs, xs, rc);
    mg(G, l + 1, rc, xc);
    prolong(G, l, xc, xs);
    symgs(G, l, rs, xs);
}

template <typename F>
std::vector<double*> vecs(Group& G, F&& f)
{
    std::vector<double*> v;
    for(auto* d : G.R) v.push_back(f(d));
    return v;
}

// The cached graph of the group's steady iteration (captured by `body` on
// first use; the cache sits in the group's first rank, keyed on the ranks'
// serial numbers, which are never reused).
template <typename F>
cudaGraphExec_t steady_graph(Group& G, bool precond, F&& body)
{
    hpcgb200_dist* d0 = G.R[0];
    std::vector<unsigned long long> key;
    for(auto* d : G.R) key.push_back(d->serial);
    if(d0->graph_exec && d0->graph_key == key && d0->graph_precond == precond) return d0->graph_exec;
    if(d0->graph_exec)
    {
        HB_HOST_CUDA(cudaStreamSynchronize(G.s));
        cudaGraphExecDestroy(d0->graph_exec);
        d0->graph_exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    HB_HOST_CUDA(cudaStreamBeginCapture(G.s, cudaStreamCaptureModeThreadLocal));
    try
    {
        body();
    }
    catch(...)
    {
        cudaStreamEndCapture(G.s, &g);
        if(g) cudaGraphDestroy(g);
        throw;
    }
    HB_HOST_CUDA(cudaStreamEndCapture(G.s, &g));
    const cudaError_t e = cudaGraphInstantiate(&d0->graph_exec, g, 0);
    cudaGraphDestroy(g);
    check_cuda(e, "cudaGraphInstantiate (decomposed CG iteration)");
    d0->graph_key = key;
    d0->graph_precond = precond;
    return d0->graph_exec;
}

// src/CG.cpp:104-200 over the group; every rank computes the same scalars.
void cg(Group& G, int max_iter, double tol, bool precond, int& niters, double& normr, double& normr0, double* hist,
        double* seconds)
{
    TraceRange trace("hpcg:CG (decomposed)");
    const auto rs = vecs(G, [](hpcgb200_dist* d) { return d->r; });
    const auto zs = vecs(G, [](hpcgb200_dist* d) { return d->z; });
    const auto ps = vecs(G, [](hpcgb200_dist* d) { return d->p; });
    const auto Aps = vecs(G, [](hpcgb200_dist* d) { return d->Ap; });
    cudaEvent_t e0, e1;
    HB_HOST_CUDA(cudaEventCreate(&e0));
    HB_HOST_CUDA(cudaEventCreate(&e1));
    HB_HOST_CUDA(cudaEventRecord(e0, G.s));
    each(G, [&](hpcgb200_dist* d, int) {
        HB_HOST_CUDA(cudaMemsetAsync(d->x, 0, sizeof(double) * d->L[0].ncols, G.s));
        HB_HOST_CUDA(cudaMemsetAsync(d->p, 0, sizeof(double) * d->L[0].ncols, G.s));  // p = x = 0
        return 0;
    });
    spmv(G, 0, ps, Aps);
    each(G, [&](hpcgb200_dist* d, int) {
        return hb::launch_dist_residual(d->L[0].m, d->local->b.d_values, d->Ap, d->r, d->sc, rt().ws, G.s);
    });
    allreduce(G, hb::kDistRr);
    normr = std::sqrt(read_slot(G, hb::kDistRr));
    normr0 = normr;
    if(hist) hist[0] = normr;
    // one iteration's work (src/CG.cpp:143-176), ending with r.r summed over
    // the ranks and copied to the first rank's pinned mirror
    auto iteration = [&](bool first) {
        if(precond) mg(G, 0, rs, zs);
        else
            each(G, [&](hpcgb200_dist* d, int) {
                HB_HOST_CUDA(cudaMemcpyAsync(d->z, d->r, sizeof(double) * d->L[0].m, cudaMemcpyDeviceToDevice, G.s));
                return 0;
            });
        each(G, [&](hpcgb200_dist* d, int) {
            return hb::launch_dot(d->L[0].m, d->r, d->z, rt().ws, d->sc + hb::kDistRtzNew, G.s);
        });
        allreduce(G, hb::kDistRtzNew);
        each(G, [&](hpcgb200_dist* d, int) {
            return hb::launch_dist_update_p(d->L[0].m, first ? 1 : 0, d->z, d->p, d->sc, G.s);
        });
        spmv(G, 0, ps, Aps);
        each(G, [&](hpcgb200_dist* d, int) {
            return hb::launch_dot(d->L[0].m, d->p, d->Ap, rt().ws, d->sc + hb::kDistPap, G.s);
        });
        allreduce(G, hb::kDistPap);
        each(G, [&](hpcgb200_dist* d, int) {
            return hb::launch_dist_update_xr(d->L[0].m, d->p, d->Ap, d->x, d->r, d->sc, rt().ws, G.s);
        });
        allreduce(G, hb::kDistRr);
        hpcgb200_dist* d0 = G.R[0];
        HB_HOST_CUDA(cudaMemcpyAsync(d0->h_sc + hb::kDistRr, d0->sc + hb::kDistRr, sizeof(double),
                                     cudaMemcpyDeviceToHost, G.s));
    };
    niters = 0;
    for(int k = 1; k <= max_iter && normr / normr0 > tol; ++k)
    {
        // the first iteration runs launch by launch: it differs (p = z) and it
        // makes every exchange once, so that all peer connections exist before
        // the steady iteration is captured
        if(k == 1 || !dist_graphs()) iteration(k == 1);
        else HB_HOST_CUDA(cudaGraphLaunch(steady_graph(G, precond, [&] { iteration(false); }), G.s));
        wait_stream(G);
        normr = std::sqrt(G.R[0]->h_sc[hb::kDistRr]);
        if(hist) hist[k] = normr;
        niters = k;
        if(!std::isfinite(normr)) break;
    }
    HB_HOST_CUDA(cudaEventRecord(e1, G.s));
    wait_stream(G);
    float ms = 0.f;
    HB_HOST_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if(seconds) *seconds = ms * 1e-3;
}

// ------------------------------------------------------------ set-up
template <typename T>
T* upload(const std::vector<T>& v, cudaStream_t s)
{
    T* d = dalloc<T>(v.size());
    if(!v.empty()) HB_HOST_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
    return d;
}

void setup_level(hpcgb200_dist* D, int l, const DistGeom& g, int* d_status)
{
    TraceRange trace("hpcg:SetupHalo");
    cudaStream_t s = rt().stream;
    DistLevel& Lv = D->L[l];
    Lv.A = D->local->levels[l];
    Lv.g = g;
    Lv.plan = plan_halo(g);
    const HaloPlan& P = Lv.plan;
    SparseMatrix& A = *Lv.A;
    Lv.m = A.localNumberOfRows;
    if(Lv.m != P.m) throw Error(HPCGB200_ERR_ARG, "halo plan and local level disagree");
    Lv.ncols = Lv.m + P.next;
    Lv.nsend = (int)P.send_rows.size();
    Lv.nh = (int)P.halo_rows.size();
    Lv.hw = P.halo_width;
    Lv.nnz = A.totalNumberOfNonzeros + (long long)P.halo_cols.size();
    A.localNumberOfColumns = Lv.ncols;

    // send buffer: the permuted rows of the send lists
    int* rows = upload(P.send_rows, s);
    Lv.send_perm = dalloc<int>(Lv.nsend);
    check(hb::launch_map_perm(Lv.nsend, rows, A.perm, Lv.send_perm, s));
    Lv.send_buf = dalloc<double>(Lv.nsend);
    // external columns into the ELL, compact halo arrays, b on level 0
    int* hrows = upload(P.halo_rows, s);
    int* hptr = upload(P.halo_ptr, s);
    int* hcols = upload(P.halo_cols, s);
    Lv.prow = dalloc<int>(Lv.nh);
    Lv.hcol = dalloc<int>((size_t)Lv.nh * std::max(Lv.hw, 1));
    Lv.hval = dalloc<double>((size_t)Lv.nh * std::max(Lv.hw, 1));
    check(hb::launch_halo_insert(Lv.nh, Lv.hw, Lv.m, hrows, hptr, hcols, A.perm, A.ell_col_ind, A.ell_val, Lv.prow,
                                 Lv.hcol, Lv.hval, l == 0 ? D->local->b.d_values : nullptr, d_status, s));
    // restriction: the coarse point a halo row is injected into (even local coordinates)
    if(A.Ac)
    {
        const int nx = g.nx, ny = g.ny, nxc = nx / 2, nyc = ny / 2;
        std::vector<int> cnat(P.halo_rows.size());
        for(size_t h = 0; h < P.halo_rows.size(); ++h)
        {
            const int row = P.halo_rows[h];
            const int iz = row / (nx * ny), iy = (row / nx) % ny, ix = row % nx;
            cnat[h] = (ix % 2 || iy % 2 || iz % 2) ? -1 : ((iz / 2) * nyc + iy / 2) * nxc + ix / 2;
        }
        int* dc = upload(cnat, s);
        Lv.pc = dalloc<int>(Lv.nh);
        check(hb::launch_map_perm(Lv.nh, dc, A.Ac->perm, Lv.pc, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        dfree(dc);
    }
    if(l >= 1)
    {
        Lv.xv = dalloc<double>(Lv.ncols);
        Lv.rv = dalloc<double>(Lv.m);
        HB_HOST_CUDA(cudaMemsetAsync(Lv.xv, 0, sizeof(double) * Lv.ncols, s));
    }
    HB_HOST_CUDA(cudaStreamSynchronize(s));
    dfree(rows);
    dfree(hrows);
    dfree(hptr);
    dfree(hcols);
}

void destroy(hpcgb200_dist* D)
{
    if(!D) return;
    if(rt().initialized) cudaStreamSynchronize(rt().stream);
    if(D->graph_exec) cudaGraphExecDestroy(D->graph_exec);  // before its communicator goes
    for(auto& Lv : D->L)
    {
        dfree(Lv.send_perm);
        dfree(Lv.send_buf);
        dfree(Lv.prow);
        dfree(Lv.hcol);
        dfree(Lv.hval);
        dfree(Lv.pc);
        dfree(Lv.xv);
        dfree(Lv.rv);
    }
    for(double* v : {D->x, D->p, D->z, D->r, D->Ap, D->b_gen, D->sc}) dfree(v);
    dfree(D->d_status);
    if(D->h_sc) cudaFreeHost(D->h_sc);
    if(D->comm) nccl().CommDestroy(D->comm);
    if(D->comm_stream) cudaStreamDestroy(D->comm_stream);
    for(cudaEvent_t e : {D->ev_packed, D->ev_recv, D->ev_sync})
        if(e) cudaEventDestroy(e);
    if(D->local) hpcgb200_problem_destroy(D->local);
    delete D;
}

const DistLevel* level_at(const hpcgb200_dist* d, int l)
{
    if(!d || l < 0 || l >= (int)d->L.size()) return nullptr;
    return &d->L[l];
}

template <typename T>
int copy_vec(const std::vector<T>& v, void* host, size_t bytes)
{
    if(bytes != v.size() * sizeof(T))
        return hb::record_error(HPCGB200_ERR_ARG, "%zu bytes requested, %zu available", bytes, v.size() * sizeof(T));
    if(bytes) std::memcpy(host, v.data(), bytes);
    return 0;
}

// Host fields of a halo plan.
int plan_field(const HaloPlan& P, const std::string& f, void* host, size_t bytes, bool& found)
{
    found = true;
    if(f == "nbr_rank") return copy_vec(P.nbr_rank, host, bytes);
    if(f == "nbr_slot") return copy_vec(P.nbr_slot, host, bytes);
    if(f == "recv_len") return copy_vec(P.recv_len, host, bytes);
    if(f == "recv_off") return copy_vec(P.recv_off, host, bytes);
    if(f == "send_len") return copy_vec(P.send_len, host, bytes);
    if(f == "send_off") return copy_vec(P.send_off, host, bytes);
    if(f == "recv_gid") return copy_vec(P.recv_gid, host, bytes);
    if(f == "send_rows") return copy_vec(P.send_rows, host, bytes);
    if(f == "halo_rows") return copy_vec(P.halo_rows, host, bytes);
    if(f == "halo_ptr") return copy_vec(P.halo_ptr, host, bytes);
    if(f == "halo_cols") return copy_vec(P.halo_cols, host, bytes);
    found = false;
    return 0;
}

void plan_info(const DistGeom& g, const HaloPlan& P, int* out)
{
    out[0] = P.m;
    out[1] = P.next;
    out[2] = (int)P.nbr_rank.size();
    out[3] = (int)P.send_rows.size();
    out[4] = (int)P.halo_rows.size();
    out[5] = P.halo_width;
    out[6] = (int)P.halo_cols.size();
    out[7] = g.npx, out[8] = g.npy, out[9] = g.npz;
    out[10] = g.ipx, out[11] = g.ipy, out[12] = g.ipz;
    out[13] = g.nx, out[14] = g.ny, out[15] = g.nz;
}

}  // namespace
}  // namespace hpcg_b200

// ------------------------------------------------------------------ C ABI

extern "C" int hpcgb200_dist_shape(int size, int* npx, int* npy, int* npz)
{
    if(!npx || !npy || !npz) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    if(size < 1) return hb::record_error(HPCGB200_ERR_ARG, "size < 1");
    optimal_shape(size, *npx, *npy, *npz);
    return 0;
}

extern "C" int hpcgb200_geometry(int size, int rank, int pz, int zl, int zu, int nx, int ny, int nz, int npx, int npy,
                                 int npz, long long* out)
{
    if(!out || size < 1 || rank < 0 || rank >= size) return hb::record_error(HPCGB200_ERR_ARG, "bad argument");
    Geometry g{};
    GenerateGeometry(size, rank, 1, pz, zl, zu, nx, ny, nz, npx, npy, npz, &g);
    const long long v[13] = {g.npx, g.npy, g.npz, g.ipx, g.ipy, g.ipz, g.gnx, g.gny, g.gnz, g.gix0, g.giy0, g.giz0,
                             g.npartz};
    std::memcpy(out, v, sizeof(v));
    DeleteGeometry(g);
    return 0;
}

extern "C" int hpcgb200_halo_plan_create(int nx, int ny, int nz, int size, int rank, int npx, int npy, int npz,
                                         hpcgb200_halo_plan** out)
{
    if(!out) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    *out = nullptr;
    if(nx < 1 || ny < 1 || nz < 1 || (long long)nx * ny * nz > 0x7fffffffLL)
        return hb::record_error(HPCGB200_ERR_ARG, "bad local brick");
    try
    {
        if(npx <= 0 || npy <= 0 || npz <= 0) optimal_shape(size, npx, npy, npz);
        auto* p = new hpcgb200_halo_plan;
        try
        {
            p->g = make_geom(size, rank, npx, npy, npz, nx, ny, nz);
            p->plan = plan_halo(p->g);
        }
        catch(...)
        {
            delete p;
            throw;
        }
        *out = p;
        return 0;
    }
    catch(const std::exception& e)
    {
        return hb::record_error(HPCGB200_ERR_ARG, "%s", e.what());
    }
}

extern "C" int hpcgb200_halo_plan_info(const hpcgb200_halo_plan* p, int* info)
{
    if(!p || !info) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    plan_info(p->g, p->plan, info);
    return 0;
}

extern "C" int hpcgb200_halo_plan_copy(const hpcgb200_halo_plan* p, const char* field, void* host, size_t bytes)
{
    if(!p || !field || (!host && bytes)) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    bool found = false;
    const int rc = plan_field(p->plan, field, host, bytes, found);
    if(!found) return hb::record_error(HPCGB200_ERR_ARG, "no plan field '%s'", field);
    return rc;
}

extern "C" int hpcgb200_halo_plan_destroy(hpcgb200_halo_plan* p)
{
    delete p;
    return 0;
}

extern "C" int hpcgb200_dist_create(int nx, int ny, int nz, int nlevels, int size, int rank, int npx, int npy,
                                    int npz, hpcgb200_dist** out)
{
    if(!out) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    *out = nullptr;
    if(size < 1 || rank < 0 || rank >= size) return hb::record_error(HPCGB200_ERR_ARG, "bad size/rank");
    if(npx <= 0 || npy <= 0 || npz <= 0) optimal_shape(size, npx, npy, npz);
    if(npx * npy * npz != size) return hb::record_error(HPCGB200_ERR_ARG, "process grid does not match size");
    static std::atomic<unsigned long long> next_serial{1};
    auto* D = new hpcgb200_dist;
    D->size = size;
    D->rank = rank;
    D->serial = next_serial++;
    int rc = hpcgb200_problem_create(nx, ny, nz, nlevels, &D->local);
    if(rc)
    {
        delete D;
        return rc;
    }
    rc = guarded([&] {
        cudaStream_t s = rt().stream;
        D->d_status = dalloc<int>(1);
        HB_HOST_CUDA(cudaMemsetAsync(D->d_status, 0, sizeof(int), s));
        D->L.resize(D->local->levels.size());
        DistGeom g = make_geom(size, rank, npx, npy, npz, nx, ny, nz);
        for(size_t l = 0; l < D->L.size(); ++l)
        {
            setup_level(D, (int)l, g, D->d_status);
            if(l + 1 < D->L.size()) g = coarsen(g);
        }
        int st = 0;
        HB_HOST_CUDA(cudaMemcpy(&st, D->d_status, sizeof(int), cudaMemcpyDeviceToHost));
        if(st) return hb::record_error(HPCGB200_ERR_DEVICE_STATUS, "external columns did not fit the ELL (%d)", st);
        const DistLevel& L0 = D->L[0];
        D->x = dalloc<double>(L0.ncols);
        D->p = dalloc<double>(L0.ncols);
        D->z = dalloc<double>(L0.ncols);
        D->r = dalloc<double>(L0.m);
        D->Ap = dalloc<double>(L0.m);
        for(double* v : {D->x, D->p, D->z}) HB_HOST_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * L0.ncols, s));
        D->b_gen = dalloc<double>(L0.m);
        HB_HOST_CUDA(cudaMemcpyAsync(D->b_gen, D->local->b.d_values, sizeof(double) * L0.m, cudaMemcpyDeviceToDevice, s));
        HB_HOST_CUDA(cudaMemcpyAsync(D->local->b_generated, D->local->b.d_values, sizeof(double) * L0.m,
                                     cudaMemcpyDeviceToDevice, s));
        D->sc = dalloc<double>(hb::kDistSlots);
        HB_HOST_CUDA(cudaMemsetAsync(D->sc, 0, sizeof(double) * hb::kDistSlots, s));
        HB_HOST_CUDA(cudaMallocHost(&D->h_sc, sizeof(double) * hb::kDistSlots));
        HB_HOST_CUDA(cudaEventCreateWithFlags(&D->ev_packed, cudaEventDisableTiming));
        HB_HOST_CUDA(cudaEventCreateWithFlags(&D->ev_recv, cudaEventDisableTiming));
        HB_HOST_CUDA(cudaEventCreateWithFlags(&D->ev_sync, cudaEventDisableTiming));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    });
    if(rc)
    {
        destroy(D);
        return rc;
    }
    *out = D;
    return 0;
}

extern "C" int hpcgb200_dist_destroy(hpcgb200_dist* d)
{
    destroy(d);
    return 0;
}

extern "C" int hpcgb200_dist_info(const hpcgb200_dist* d, int level, int* info, long long* nnz)
{
    const DistLevel* Lv = level_at(d, level);
    if(!Lv || !info) return hb::record_error(HPCGB200_ERR_ARG, "bad level or null argument");
    plan_info(Lv->g, Lv->plan, info);
    info[16] = d->size;
    info[17] = d->rank;
    info[18] = (int)d->L.size();
    info[19] = Lv->A->nblocks;
    if(nnz) *nnz = Lv->nnz;
    return 0;
}

extern "C" int hpcgb200_dist_copy_field(const hpcgb200_dist* d, int level, const char* field, void* host,
                                        size_t bytes)
{
    const DistLevel* Lv = level_at(d, level);
    if(!Lv || !field || (!host && bytes)) return hb::record_error(HPCGB200_ERR_ARG, "bad level or null argument");
    bool found = false;
    int rc = plan_field(Lv->plan, field, host, bytes, found);
    if(found) return rc;
    return guarded([&] {
        const std::string f = field;
        const SparseMatrix& A = *Lv->A;
        const size_t m = (size_t)Lv->m;
        const void* src = nullptr;
        size_t n = 0;
        if(f == "ell_col") src = A.ell_col_ind, n = m * 27 * 4;
        else if(f == "ell_val") src = A.ell_val, n = m * 27 * 8;
        else if(f == "perm") src = A.perm, n = m * 4;
        else if(f == "send_perm") src = Lv->send_perm, n = (size_t)Lv->nsend * 4;
        else if(f == "halo_prow") src = Lv->prow, n = (size_t)Lv->nh * 4;
        else if(f == "halo_col") src = Lv->hcol, n = (size_t)Lv->nh * Lv->hw * 4;
        else if(f == "halo_pc" && Lv->pc) src = Lv->pc, n = (size_t)Lv->nh * 4;
        else if(level == 0 && f == "b") src = d->local->b.d_values, n = m * 8;
        else if(level == 0 && f == "x") src = d->x, n = (size_t)Lv->ncols * 8;
        else return hb::record_error(HPCGB200_ERR_ARG, "no field '%s' on level %d", field, level);
        if(bytes != n)
            return hb::record_error(HPCGB200_ERR_ARG, "field '%s': %zu bytes requested, %zu available", field, bytes, n);
        HB_HOST_CUDA(cudaStreamSynchronize(rt().stream));
        if(n) HB_HOST_CUDA(cudaMemcpy(host, src, n, cudaMemcpyDeviceToHost));
        return 0;
    });
}

extern "C" int hpcgb200_dist_nccl_available(void)
{
    return nccl().ok ? 1 : 0;
}

extern "C" int hpcgb200_dist_nccl_id(void* id, size_t bytes)
{
    if(!id || bytes != sizeof(ncclUniqueId))
        return hb::record_error(HPCGB200_ERR_ARG, "id needs %zu bytes", sizeof(ncclUniqueId));
    NcclApi& N = nccl();
    if(!N.ok) return hb::record_error(HPCGB200_ERR_COMM, "NCCL unavailable: %s", N.why.c_str());
    try
    {
        ncclUniqueId u;
        check_nccl(N.GetUniqueId(&u), "ncclGetUniqueId");
        std::memcpy(id, &u, sizeof(u));
        return 0;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

extern "C" int hpcgb200_dist_attach_nccl(hpcgb200_dist* d, const void* id, size_t bytes)
{
    if(!d || !id || bytes != sizeof(ncclUniqueId)) return hb::record_error(HPCGB200_ERR_ARG, "bad argument");
    NcclApi& N = nccl();
    if(!N.ok) return hb::record_error(HPCGB200_ERR_COMM, "NCCL unavailable: %s", N.why.c_str());
    return guarded([&] {
        if(d->comm) return hb::record_error(HPCGB200_ERR_ARG, "communicator already attached");
        ncclUniqueId u;
        std::memcpy(&u, id, sizeof(u));
        check_nccl(N.CommInitRank(&d->comm, d->size, u, d->rank), "ncclCommInitRank");
        HB_HOST_CUDA(cudaStreamCreateWithFlags(&d->comm_stream, cudaStreamNonBlocking));
        return 0;
    });
}

extern "C" int hpcgb200_dist_set_rhs(hpcgb200_dist* d, const double* host_b_natural)
{
    if(!d) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        const int m = d->L[0].m;
        cudaStream_t s = rt().stream;
        if(!host_b_natural)
            HB_HOST_CUDA(cudaMemcpyAsync(d->local->b.d_values, d->b_gen, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        else
        {
            double* tmp = opt(*d->local->levels[0])->vec_scratch;
            HB_HOST_CUDA(cudaMemcpyAsync(tmp, host_b_natural, sizeof(double) * m, cudaMemcpyHostToDevice, s));
            check(hpcgb200_permute_vector(m, d->local->A.perm, tmp, d->local->b.d_values, s));
        }
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    });
}

extern "C" int hpcgb200_dist_get_x(hpcgb200_dist* d, double* host_x_natural)
{
    if(!d || !host_x_natural) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        const int m = d->L[0].m;
        cudaStream_t s = rt().stream;
        double* tmp = opt(*d->local->levels[0])->vec_scratch;
        check(hpcgb200_unpermute_vector(m, d->local->A.perm, d->x, tmp, s));
        HB_HOST_CUDA(cudaMemcpyAsync(host_x_natural, tmp, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    });
}

extern "C" int hpcgb200_dist_group_spmv(hpcgb200_dist* const* ranks, int n, int level, double* const* x,
                                        double* const* y)
{
    if(!x || !y) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        Group G = make_group(ranks, n);
        if(level < 0 || level >= G.nlevels) return hb::record_error(HPCGB200_ERR_ARG, "bad level");
        spmv(G, level, std::vector<double*>(x, x + n), std::vector<double*>(y, y + n));
        wait_stream(G);
        return 0;
    });
}

extern "C" int hpcgb200_dist_group_symgs(hpcgb200_dist* const* ranks, int n, int level, double* const* r,
                                         double* const* x)
{
    if(!r || !x) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        Group G = make_group(ranks, n);
        if(level < 0 || level >= G.nlevels) return hb::record_error(HPCGB200_ERR_ARG, "bad level");
        symgs(G, level, std::vector<double*>(r, r + n), std::vector<double*>(x, x + n));
        wait_stream(G);
        return 0;
    });
}

extern "C" int hpcgb200_dist_group_restrict(hpcgb200_dist* const* ranks, int n, int level, double* const* rf,
                                            double* const* xf, double* const* rc)
{
    if(!rf || !xf || !rc) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        Group G = make_group(ranks, n);
        if(level < 0 || level + 1 >= G.nlevels) return hb::record_error(HPCGB200_ERR_ARG, "bad level");
        restrict_fused(G, level, std::vector<double*>(rf, rf + n), std::vector<double*>(xf, xf + n),
                       std::vector<double*>(rc, rc + n));
        wait_stream(G);
        return 0;
    });
}

extern "C" int hpcgb200_dist_group_mg(hpcgb200_dist* const* ranks, int n, double* const* r, double* const* x)
{
    if(!r || !x) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        Group G = make_group(ranks, n);
        mg(G, 0, std::vector<double*>(r, r + n), std::vector<double*>(x, x + n));
        wait_stream(G);
        return 0;
    });
}

extern "C" int hpcgb200_dist_group_cg(hpcgb200_dist* const* ranks, int n, int max_iter, double tol, int precond,
                                      int* niters, double* normr, double* normr0, double* normr_hist, double* seconds)
{
    if(!niters || !normr || !normr0) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    if(max_iter < 0) return hb::record_error(HPCGB200_ERR_ARG, "max_iter < 0");
    return guarded([&] {
        Group G = make_group(ranks, n);
        cg(G, max_iter, tol, precond != 0, *niters, *normr, *normr0, normr_hist, seconds);
        if(!std::isfinite(*normr) || !std::isfinite(*normr0))
            return hb::record_error(HPCGB200_ERR_NONFINITE, "decomposed CG ended with a non-finite residual");
        return 0;
    });
}

extern "C" int hpcgb200_dist_cg(hpcgb200_dist* d, int max_iter, double tol, int precond, int* niters, double* normr,
                                double* normr0, double* normr_hist, double* seconds)
{
    return hpcgb200_dist_group_cg(&d, 1, max_iter, tol, precond, niters, normr, normr0, normr_hist, seconds);
}
