// CG (src/CG.cpp:104-200) as a device-resident loop.
//
// The preamble (p = x, Ap = A p, r = b - Ap, normr0) runs as plain launches
// followed by one read-back.  The iterations are one CUDA graph: a
// conditional WHILE node whose body is MG (or z = r), rtz, p update, SpMV+pAp,
// r/x update; the last kernel of the body evaluates the reference's loop
// condition (k <= max_iter && normr/normr0 > tol) on the device and feeds it
// to the WHILE node.  A solve therefore costs one graph launch and two
// read-backs instead of the reference's 12 device syncs + 3 blocking copies
// per iteration.  Where conditional nodes are unavailable the same body runs
// as a per-iteration graph with a host-side check.
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "hpcg_b200.h"
#include "internal.hpp"
#include "learned.hpp"

using namespace hpcg_b200;

namespace hpcg_b200 {

static void ensure_state(LevelOpt* o, int max_iter)
{
    if(!o->step_barrier) o->step_barrier = dalloc<hb::GridBarrier>(1);
    if(o->cg_state && o->cg_state_iters >= max_iter) return;
    const int cap = max_iter < 1024 ? 1024 : max_iter;
    dfree(o->cg_state);
    o->cg_state = reinterpret_cast<hb::CGState*>(dalloc<char>(hb::cg_state_bytes(cap)));
    o->cg_state_iters = cap;
    // graphs captured the old state pointer
    for(auto& g : o->graphs)
    {
        if(g->exec) cudaGraphExecDestroy(g->exec);
        if(g->graph) cudaGraphDestroy(g->graph);
    }
    o->graphs.clear();
}

// The CG step after the preconditioner as two kernels (rtz + p update + SpMV
// + pAp, then r/x update + normr + loop control) or five (rtz, p update,
// SpMV + pAp, r/x update, loop control).  Measured on B200 (A/B on one box):
// mixed 320^3 0.3800 vs 0.3826 s, so the FP32 V-cycle modes take two by
// default; FP64 ELL 256^3 0.6889 vs 0.6893 s, a wash, so it keeps five, whose
// reduction partitions the FP64 stencil mode shares for its bit-identical
// history.  HPCGB200_CG_STEP=2 / =5 selects two / five kernels for every mode
// that has both (untimed bodies only; the phase-timed body keeps five).
static bool cg_step2_for(MGPrecision prec)
{
    static const int forced = [] {
        const char* e = std::getenv("HPCGB200_CG_STEP");
        return e && e[0] == '2' ? 2 : (e && e[0] == '5' ? 5 : 0);
    }();
    if(forced) return forced == 2;
    return prec == MGPrecision::FP32 || prec == MGPrecision::LEARNED;
}

// timed: phase timers around the operators (reference times[] slots: MG,
// r.z -> dot, p update -> WAXPBY, SpMV with p.Ap -> SpMV, r/x update with
// ||r|| -> WAXPBY).
static int capture_body(const SparseMatrix& A, CGData& data, Vector& x, bool precond, MGPrecision prec,
                        hb::CGState* st, unsigned long long cond, cudaStream_t s, bool timed = false)
{
    const int n = A.localNumberOfRows;
    auto stamp = [&](int phase) { return timed ? hb::launch_cg_timer(st, phase, s) : 0; };
    HB_RETURN_IF(stamp(hb::kPhaseStart));
    // the FP32 V-cycles' output is read in FP32 by the CG kernels (z32)
    const float* z32 = nullptr;
    if(precond)
    {
        if(prec == MGPrecision::FP64) HB_RETURN_IF(ComputeMG(A, data.r, data.z));
        else if(prec == MGPrecision::FP64_STENCIL) HB_RETURN_IF(ComputeMG_Stencil(A, data.r, data.z));
        else
        {
            if(prec == MGPrecision::FP32) HB_RETURN_IF(mg_mixed_to(A, data.r.d_values, nullptr, s));
            else HB_RETURN_IF(mg_learned_to(A, data.r.d_values, nullptr, s));
            z32 = opt(A)->z32;
        }
    }
    else
    {
        const cudaError_t e =
            cudaMemcpyAsync(data.z.d_values, data.r.d_values, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        if(e != cudaSuccess) return hb::cuda_error(e, "copy r to z", __FILE__, __LINE__);
    }
    HB_RETURN_IF(stamp(hb::kPhaseMG));
    const int watch = prec == MGPrecision::LEARNED ? 1 : 0;
    if(!timed && cg_step2_for(prec) && (prec == MGPrecision::FP64 || z32))
    {
        LevelOpt* o = opt(A);
        if(z32)
            HB_RETURN_IF(hb::launch_cg_step1_sep(o->st, o->diag, data.r.d_values, z32, data.p.d_values, x.d_values,
                                                 data.Ap.d_values, st, rt().ws, o->step_barrier, s));
        else
            HB_RETURN_IF(hb::launch_cg_step1_ell(n, o->cc, A.ell_col_ind, A.ell_val, data.r.d_values,
                                                 data.z.d_values, data.p.d_values, x.d_values, data.Ap.d_values, st,
                                                 rt().ws, o->step_barrier, s));
        return z32 ? hb::launch_cg_step2(n, data.Ap.d_values, data.r.d_values, z32, st, rt().ws, cond, watch, s)
                   : hb::launch_cg_step2(n, data.Ap.d_values, data.r.d_values, data.z.d_values, st, rt().ws, cond,
                                         watch, s);
    }
    HB_RETURN_IF(z32 ? hb::launch_cg_rtz(n, data.r.d_values, z32, st, rt().ws, s)
                     : hb::launch_cg_rtz(n, data.r.d_values, data.z.d_values, st, rt().ws, s));
    HB_RETURN_IF(stamp(hb::kPhaseDot));
    HB_RETURN_IF(z32 ? hb::launch_cg_update_p(n, z32, data.p.d_values, x.d_values, st, s)
                     : hb::launch_cg_update_p(n, data.z.d_values, data.p.d_values, x.d_values, st, s));
    HB_RETURN_IF(stamp(hb::kPhaseWaxpby));
    if(prec == MGPrecision::FP64_STENCIL)
    {
        // the implicit-stencil product, then p.Ap with the ELL kernel's partition: the FP64 path's scalars
        const LevelOpt* o = opt(A);
        HB_RETURN_IF(hb::launch64_spmv_stencil(o->st, o->diag, data.p.d_values, data.Ap.d_values, s));
        HB_RETURN_IF(hb::launch_cg_pap_chunks(n, o->cc, data.p.d_values, data.Ap.d_values, st, o->spmv_partial,
                                              o->spmv_ticket, s));
    }
    else if(prec != MGPrecision::FP64)
    {
        // mixed path: the FP64 operator on the implicit stencil (separable sum, equal to the ELL product to
        // FP64 rounding)
        const LevelOpt* o = opt(A);
        HB_RETURN_IF(hb::launch64_cg_spmv_pap_stencil(o->st, o->diag, data.p.d_values, data.Ap.d_values, st,
                                                      o->pap_partial, o->pap_ticket, s));
    }
    else
    {
        const LevelOpt* o = opt(A);
        HB_RETURN_IF(hb::launch_cg_spmv_pap(n, o->cc, A.ell_col_ind, A.ell_val, data.p.d_values, data.Ap.d_values, st,
                                            o->spmv_partial, o->spmv_ticket, s));
    }
    HB_RETURN_IF(stamp(hb::kPhaseSpmv));
    HB_RETURN_IF(z32 ? hb::launch_cg_update_r(n, data.Ap.d_values, data.r.d_values, z32, st, rt().ws, cond, watch, s)
                     : hb::launch_cg_update_r(n, data.Ap.d_values, data.r.d_values, data.z.d_values, st, rt().ws,
                                              cond, watch, s));
    // (the r update kernel launches the loop control after itself; its
    // stamp below also covers that one-thread kernel)
    HB_RETURN_IF(stamp(hb::kPhaseWaxpby));
    return 0;
}

static int count_kernel_nodes(cudaGraph_t g)
{
    size_t n = 0;
    if(cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if(cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    int k = 0;
    for(auto nd : nodes)
    {
        cudaGraphNodeType t;
        if(cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    return k;
}

static CGGraph* get_graph(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, bool precond,
                          MGPrecision prec, bool flexible, bool timed = false)
{
    LevelOpt* o = opt(A);
    const double* key[6] = {data.r.d_values, data.z.d_values, data.p.d_values, data.Ap.d_values, b.d_values,
                            x.d_values};
    const void* sm = prec == MGPrecision::LEARNED ? o->smoother : nullptr;
    const long long sm_epoch = sm ? o->smoother->epoch : -1;
    for(auto it = o->graphs.begin(); it != o->graphs.end(); ++it)
    {
        CGGraph* g = it->get();
        if(std::memcmp(g->key, key, sizeof(key)) || g->mode != (int)prec || g->precond != precond ||
           g->flexible != flexible || g->timed != timed)
            continue;
        if(g->smoother == sm && g->smoother_epoch == sm_epoch) return g;
        if(g->exec) cudaGraphExecDestroy(g->exec);  // captured other smoother buffers
        if(g->graph) cudaGraphDestroy(g->graph);
        o->graphs.erase(it);
        break;
    }

    auto G = std::make_unique<CGGraph>();
    std::memcpy(G->key, key, sizeof(key));
    G->mode = (int)prec;
    G->precond = precond;
    G->flexible = flexible;
    G->timed = timed;
    G->smoother = sm;
    G->smoother_epoch = sm_epoch;
    cudaStream_t s = rt().stream;

    // Preferred: WHILE conditional node around the iteration body.
    bool built = false;
    {
        cudaGraph_t g = nullptr;
        cudaGraphConditionalHandle h = 0;
        cudaGraphNode_t node;
        cudaGraphNodeParams cp{};
        if(cudaGraphCreate(&g, 0) == cudaSuccess &&
           cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess)
        {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            if(cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess)
            {
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                if(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                   cudaSuccess)
                {
                    const int rc =
                        capture_body(A, data, x, precond, prec, o->cg_state, (unsigned long long)h, s, timed);
                    cudaGraph_t out = nullptr;
                    const cudaError_t e = cudaStreamEndCapture(s, &out);
                    if(rc == 0 && e == cudaSuccess && cudaGraphInstantiate(&G->exec, g, 0) == cudaSuccess)
                    {
                        G->kernels_per_iteration = count_kernel_nodes(body);
                        G->graph = g;
                        G->conditional = true;
                        built = true;
                    }
                }
            }
        }
        if(!built)
        {
            cudaGetLastError();
            if(g) cudaGraphDestroy(g);
        }
    }
    if(!built)
    {
        // Fallback: one iteration per launch, host checks the condition.
        cudaGraph_t g = nullptr;
        HB_HOST_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int rc = capture_body(A, data, x, precond, prec, o->cg_state, 0ULL, s, timed);
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        if(rc) throw_last(rc);
        HB_HOST_CUDA(e);
        HB_HOST_CUDA(cudaGraphInstantiate(&G->exec, g, 0));
        G->kernels_per_iteration = count_kernel_nodes(g);
        G->graph = g;
        G->conditional = false;
    }
    o->graphs.push_back(std::move(G));
    return o->graphs.back().get();
}

int iteration_kernels(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, bool precond,
                      MGPrecision prec, bool flexible)
{
    LevelOpt* o = opt(A);
    ensure_state(o, 1);
    if(prec == MGPrecision::LEARNED)
    {
        if(!o->smoother) throw Error(HPCGB200_ERR_ARG, "learned CG: no smoother attached to the problem");
        check(smoother_ready(A, rt().stream));
    }
    return get_graph(A, data, b, x, precond, prec, flexible)->kernels_per_iteration;
}

// HPCGB200_GRAPH=0 runs the iteration body as direct launches with a host
// check per iteration (for profilers that cannot look inside graphs with
// conditional nodes); the kernels and their order are the same.
static bool graphs_enabled()
{
    const char* e = std::getenv("HPCGB200_GRAPH");
    return !(e && e[0] == '0');
}

int run_cg(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, int max_iter, double tol, int& niters,
           double& normr, double& normr0, bool precond, MGPrecision prec, bool flexible, double* hist,
           double* seconds, double* phase_seconds)
{
    const bool timed = phase_seconds != nullptr;
    TraceRange trace("hpcg:CG");
    try
    {
        ensure_runtime();
        if(max_iter < 0 || max_iter > 1000000) return hb::record_error(HPCGB200_ERR_ARG, "CG: max_iter out of range");
        LevelOpt* o = opt(A);
        if(!o) return hb::record_error(HPCGB200_ERR_ARG, "CG: OptimizeProblem has not run");
        cudaStream_t s = rt().stream;
        const int n = A.localNumberOfRows;
        ensure_state(o, max_iter);
        hb::CGState* st = o->cg_state;

        hb::CGState h{};
        h.tol = tol;
        h.max_iter = max_iter;
        h.flexible = flexible ? 1 : 0;
        h.net = prec == MGPrecision::LEARNED ? 1 : 0;
        h.fb_jump = o->fb_jump;
        h.fb_rate = o->fb_rate;
        h.fb_stall = o->fb_stall;
        h.fb_window = o->fb_window;
        if(prec == MGPrecision::LEARNED && !o->smoother)
            return hb::record_error(HPCGB200_ERR_ARG, "learned CG: no smoother attached to the problem");
        if(prec == MGPrecision::LEARNED) check(smoother_ready(A, s));
        cudaEvent_t e0, e1;
        HB_HOST_CUDA(cudaEventCreate(&e0));
        HB_HOST_CUDA(cudaEventCreate(&e1));
        HB_HOST_CUDA(cudaEventRecord(e0, s));
        HB_HOST_CUDA(cudaMemcpyAsync(st, &h, offsetof(hb::CGState, hist), cudaMemcpyHostToDevice, s));
        // fresh reduction tickets and grid barrier for every solve
        HB_HOST_CUDA(cudaMemsetAsync(&rt().ws->ticket, 0, sizeof(unsigned int), s));
        HB_HOST_CUDA(cudaMemsetAsync(o->step_barrier, 0, sizeof(hb::GridBarrier), s));
        if(o->pap_ticket) HB_HOST_CUDA(cudaMemsetAsync(o->pap_ticket, 0, sizeof(unsigned int), s));
        HB_HOST_CUDA(cudaMemsetAsync(o->spmv_ticket, 0, sizeof(unsigned int), s));

        // the FP32 V-cycles need the stencil on every level; the FP64 stencil
        // V-cycle takes the ELL kernels on levels without it, only the outer
        // SpMV needs it on level 0
        if(prec != MGPrecision::FP64)
            for(const SparseMatrix* M = &A; M; M = prec == MGPrecision::FP64_STENCIL ? nullptr : M->Ac)
                if(!opt(*M) || !opt(*M)->stencil_ok)
                    return hb::record_error(HPCGB200_ERR_NOT_STENCIL,
                                            "stencil CG needs the 27-point stencil in parity colouring on every level");
        // preamble: p = x; Ap = A p; r = b - Ap; normr = ||r|| (resets the
        // device iteration counter and the history)
        auto preamble = [&] {
            HB_HOST_CUDA(cudaMemcpyAsync(data.p.d_values, x.d_values, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                         s));
            if(prec != MGPrecision::FP64)
                check(hb::launch64_spmv_stencil(o->st, o->diag, data.p.d_values, data.Ap.d_values, s));
            else
                check(hb::launch_spmv(n, o->cc, A.ell_col_ind, A.ell_val, data.p.d_values, data.Ap.d_values, s));
            check(hb::launch_cg_residual0(n, b.d_values, data.Ap.d_values, data.r.d_values, st, rt().ws, s));
            HB_HOST_CUDA(cudaMemcpyAsync(&h, st, offsetof(hb::CGState, hist), cudaMemcpyDeviceToHost, s));
            HB_HOST_CUDA(cudaStreamSynchronize(s));
        };
        // learned mode: keep the initial guess, so that a network step that
        // makes the residual non-finite costs a restart, not the solution
        if(prec == MGPrecision::LEARNED)
        {
            if(!o->x0_saved) o->x0_saved = dalloc<double>(n);
            HB_HOST_CUDA(cudaMemcpyAsync(o->x0_saved, x.d_values, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        }
        preamble();
        int restart_offset = 0;            // iterations spent before a restart
        std::vector<double> hist_before;   // their residual history

        // Iterations: the learned mode runs until converged or until its
        // smoother fails (a jump or a stall of normr); the plain FP32 V-cycle then takes
        // over from the same state (flexible CG tolerates the switch).
        MGPrecision cur = prec;
        for(int phase = 0; phase < 2; ++phase)
        {
            const bool iterate = h.k <= max_iter && max_iter >= 1 && (h.normr / h.normr0 > tol);
            if(!iterate) break;
            if(!graphs_enabled())
            {
                for(int k = h.k; k <= max_iter - restart_offset; ++k)
                {
                    check(capture_body(A, data, x, precond, cur, st, 0ULL, s, timed));
                    HB_HOST_CUDA(cudaMemcpyAsync(&h, st, offsetof(hb::CGState, hist), cudaMemcpyDeviceToHost, s));
                    HB_HOST_CUDA(cudaStreamSynchronize(s));
                    if(!(h.normr / h.normr0 > tol) || (cur == MGPrecision::LEARNED && h.net == 2)) break;
                }
            }
            else
            {
                CGGraph* G = get_graph(A, data, b, x, precond, cur, flexible, timed);
                if(G->conditional)
                {
                    HB_HOST_CUDA(cudaGraphLaunch(G->exec, s));
                }
                else
                {
                    for(int k = h.k; k <= max_iter - restart_offset; ++k)
                    {
                        HB_HOST_CUDA(cudaGraphLaunch(G->exec, s));
                        HB_HOST_CUDA(cudaMemcpyAsync(&h, st, offsetof(hb::CGState, hist), cudaMemcpyDeviceToHost, s));
                        HB_HOST_CUDA(cudaStreamSynchronize(s));
                        if(!(h.normr / h.normr0 > tol) || (cur == MGPrecision::LEARNED && h.net == 2)) break;
                    }
                }
            }
            HB_HOST_CUDA(cudaMemcpyAsync(&h, st, offsetof(hb::CGState, hist), cudaMemcpyDeviceToHost, s));
            HB_HOST_CUDA(cudaStreamSynchronize(s));
            if(cur != MGPrecision::LEARNED || h.net != 2) break;
            cur = MGPrecision::FP32;
            if(!std::isfinite(h.normr))
            {
                // the network's step poisoned x and r: restart the plain
                // FP32 V-cycle solve from the initial guess, keeping the
                // abandoned iterations in the count and the history
                restart_offset = h.niters;
                hist_before.resize(restart_offset + 1);
                HB_HOST_CUDA(cudaMemcpy(hist_before.data(), st->hist, sizeof(double) * (restart_offset + 1),
                                        cudaMemcpyDeviceToHost));
                HB_HOST_CUDA(cudaMemcpyAsync(x.d_values, o->x0_saved, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                             s));
                const int left = max_iter - restart_offset;
                HB_HOST_CUDA(cudaMemcpyAsync(&st->max_iter, &left, sizeof(int), cudaMemcpyHostToDevice, s));
                // a fresh solve: no pending direction restart (the fallback
                // iteration is reported from restart_offset)
                const int none = 0;
                HB_HOST_CUDA(cudaMemcpyAsync(&st->fallback_iter, &none, sizeof(int), cudaMemcpyHostToDevice, s));
                preamble();
                if(left < 1) break;
            }
        }
        // the last iteration's x += alpha p (each iteration's update runs in
        // the next iteration's p update)
        check(hb::launch_cg_x_final(n, data.p.d_values, x.d_values, st, s));
        HB_HOST_CUDA(cudaEventRecord(e1, s));
        HB_HOST_CUDA(cudaMemcpyAsync(&h, st, offsetof(hb::CGState, hist), cudaMemcpyDeviceToHost, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        float ms = 0.f;
        HB_HOST_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if(hist)
        {
            // after a restart: the abandoned iterations, then the restarted
            // solve's iterations 1.. (its normr0 is the same)
            for(int k = 0; k <= restart_offset && restart_offset > 0; ++k) hist[k] = hist_before[k];
            HB_HOST_CUDA(cudaMemcpy(hist + restart_offset + (restart_offset > 0), st->hist + (restart_offset > 0),
                                    sizeof(double) * (h.niters + 1 - (restart_offset > 0)), cudaMemcpyDeviceToHost));
            for(int k = restart_offset + h.niters + 1; k <= max_iter; ++k) hist[k] = 0.0;
        }
        if(h.status)
            return hb::record_error(HPCGB200_ERR_DEVICE_STATUS,
                                    "CG: a bounded device wait of the CG step timed out (status %d: 1 grid barrier, "
                                    "3 TMA copies)",
                                    h.status);
        for(const SparseMatrix* M = &A; M; M = M->Ac)
        {
            const LevelOpt* lo = opt(*M);
            if(!lo || !lo->pass_status) continue;
            int ps = 0;
            HB_HOST_CUDA(cudaMemcpy(&ps, lo->pass_status, sizeof(int), cudaMemcpyDeviceToHost));
            if(ps)
                return hb::record_error(HPCGB200_ERR_DEVICE_STATUS,
                                        "CG: the copies of a TMA-staged colour pass timed out (status %d)", ps);
        }
        o->last_fallback_iter = restart_offset > 0 ? restart_offset : h.fallback_iter;
        if(prec == MGPrecision::LEARNED) check(smoother_status(*o->smoother, s));
        niters = restart_offset + h.niters;
        normr = h.normr;
        normr0 = h.normr0;
        if(seconds) *seconds = ms * 1e-3;
        if(phase_seconds)
            for(int q = 0; q < 4; ++q) phase_seconds[q] = h.phase_ns[q] * 1e-9;
        return 0;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

}  // namespace hpcg_b200

int CG_B200(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, int max_iter, double tolerance,
            int& niters, double& normr, double& normr0, double* times, bool doPreconditioning, MGPrecision prec,
            bool flexible, double* normr_hist)
{
    const auto t0 = std::chrono::steady_clock::now();
    double phase[4] = {0.0, 0.0, 0.0, 0.0};
    const int rc = run_cg(A, data, b, x, max_iter, tolerance, niters, normr, normr0, doPreconditioning, prec, flexible,
                          normr_hist, nullptr, times ? phase : nullptr);
    if(times)
    {
        times[0] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        // src/CG.cpp's slots: 1 dot products, 2 WAXPBY, 3 SpMV, 5 preconditioner
        times[1] += phase[hb::kPhaseDot];
        times[2] += phase[hb::kPhaseWaxpby];
        times[3] += phase[hb::kPhaseSpmv];
        times[5] += phase[hb::kPhaseMG];
    }
    return rc;
}

int CG(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, const int max_iter, const double tolerance,
       int& niters, double& normr, double& normr0, double* times, bool doPreconditioning, bool verbose)
{
    std::vector<double> hist(verbose ? max_iter + 1 : 0);
    const int rc = CG_B200(A, data, b, x, max_iter, tolerance, niters, normr, normr0, times, doPreconditioning,
                           MGPrecision::FP64, false, verbose ? hist.data() : nullptr);
    if(rc == 0 && verbose)
    {
        printf("B200 Initial Residual = %le\n", normr0);
        for(int k = 1; k <= niters; ++k) printf("B200 Iteration = %d   Scaled Residual = %le\n", k, hist[k] / normr0);
    }
    return rc;
}
