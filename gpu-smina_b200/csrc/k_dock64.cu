// Plain (FP64) path kernels: one warp (one 32-thread block) per item.
// Built with -fmad=false so that the arithmetic rounds exactly like the
// CPU restatement compiled with -ffp-contract=off.
#include "dock64_search.cuh"

namespace sg {

__device__ void init_ws64(W64& w, const DModel* m, const DTables* T, const DReceptor* R, int* err) {
    extern __shared__ double smem64[];
    w.s = smem64;
    w.m = m;
    w.T = T;
    w.R = R;
    w.err = err;
    w.lane = threadIdx.x & 31;
    w.evals = 0;
    w.box = nullptr;
    w.L = ws64_layout(m->natoms, m->nframes, m->npairs, m->conf_size, m->dof);
    w.pin = reinterpret_cast<uint8_t*>(w.s + w.L.pin);
    w.mt = reinterpret_cast<uint32_t*>(w.s + w.L.mt);
    // model state as read: coords and frame origins (mutation reads them)
    for (int i = w.lane; i < 3 * m->natoms; i += 32) w.s[w.L.coords + i] = m->lab[i];
    for (int i = w.lane; i < 3 * m->nframes; i += 32) {
        w.s[w.L.origin + i] = m->finit[i];
        w.s[w.L.axis + i] = m->faxis[i];
    }
    for (int f = w.lane; f < m->nframes; f += 32) {
        double* q = w.s + w.L.q + 4 * f;
        q[0] = 1; q[1] = 0; q[2] = 0; q[3] = 0;
        quat_to_mat(Quat<double>{1, 0, 0, 0}, w.s + w.L.rot + 9 * f);
    }
    __syncwarp();
}

// model::eval_deriv for a batch of confs of one model
__global__ void __launch_bounds__(32) k_eval64(const DModel* model, DTables T, const DReceptor* R, int nconfs,
                                               const double* confs, double v0, double v1, double v2, double slope,
                                               int direct, double* out_e, double* out_g, double* out_coords, int* err) {
    W64 w;
    init_ws64(w, model, &T, R, err);
    const int k = blockIdx.x;
    if (k >= nconfs) return;
    const DModel& m = *model;
    double* x = w.s + w.L.x_tmp;
    vcopy(w, x, confs + (size_t)k * m.conf_size, m.conf_size);
    EvalMode em{{v0, v1, v2}, slope, direct != 0};
    double* g = w.s + w.L.g;
    const double e = feval(w, x, g, em);
    if (w.lane == 0) out_e[k] = e;
    for (int i = w.lane; i < m.dof; i += 32) out_g[(size_t)k * m.dof + i] = g[i];
    if (out_coords)
        for (int i = w.lane; i < 3 * m.nmov; i += 32) out_coords[(size_t)k * 3 * m.nmov + i] = w.s[w.L.coords + i];
}

// quasi_newton on the grid maps for a batch of confs (confs updated in place)
__global__ void __launch_bounds__(32) k_bfgs64(const DModel* model, DTables T, const DReceptor* R, int nconfs,
                                               double* confs, double v0, double v1, double v2, double slope,
                                               int maxiters, int accurate, int early, double* out_e, int* err) {
    W64 w;
    init_ws64(w, model, &T, R, err);
    const int k = blockIdx.x;
    if (k >= nconfs) return;
    const DModel& m = *model;
    double* x = w.s + w.L.x_tmp;
    vcopy(w, x, confs + (size_t)k * m.conf_size, m.conf_size);
    EvalMode em{{v0, v1, v2}, slope, false};
    const double e = bfgs64(w, x, maxiters, accurate, early, em);
    if (w.lane == 0) out_e[k] = e;
    for (int i = w.lane; i < m.conf_size; i += 32) confs[(size_t)k * m.conf_size + i] = x[i];
}

// monte_carlo::operator() for one chain per block
// VIS: chains may carry a QuickVina 2 history (a separate instantiation, so
// smina's own search compiles exactly as without it)
template <bool VIS>
__global__ void __launch_bounds__(32) k_mc64(const DModel* models, DTables T, const DReceptor* R,
                                             const Chain64* chains, int nchains, MCParams64 P, int* err) {
    const int c = blockIdx.x;
    if (c >= nchains) return;
    const Chain64 ch = chains[c];
    const DModel* mp = models + ch.model;
    W64 w;
    init_ws64(w, mp, &T, R, err);
    const DModel& m = *mp;
    for (int i = w.lane; i < 625; i += 32) w.mt[i] = ch.mt[i];
    double* tmp = w.s + w.L.x_tmp;
    double* cand = w.s + w.L.x_cand;
    vcopy(w, tmp, ch.conf0, m.conf_size);
    if (w.lane == 0) *ch.out_count = 0;
    __syncwarp();
    const EvalMode hunt{{P.hunt[0], P.hunt[1], P.hunt[2]}, P.slope, false};
    const EvalMode auth{{P.auth[0], P.auth[1], P.auth[2]}, P.slope, false};
    Hist64 hist_store{};
    const Hist64* vis = nullptr;
    if (VIS && ch.hist && m.dof <= kHistMaxN) {
        hist_store = hist64_view(ch.hist, ch.hist_words, m.dof);
        vis = &hist_store;
    }
    double tmp_e = 0, best_e = kMaxFl;
    for (unsigned step = 0; step < ch.steps; step++) {
        vcopy(w, cand, tmp, m.conf_size);
        mutate64(w, cand, P.amplitude);
        const double cand_e = bfgs64(w, cand, ch.maxiters, P.accurate_line, P.early_term, hunt, vis);
        if (step == 0 || metropolis64(w, tmp_e, cand_e, P.temperature)) {
            vcopy(w, tmp, cand, m.conf_size);
            tmp_e = cand_e;
            set_conf64(w, tmp);
            const int count = *ch.out_count;
            if (tmp_e < best_e || count < P.num_saved) {
                tmp_e = bfgs64(w, tmp, ch.maxiters, P.accurate_line, P.early_term, auth, vis);
                set_conf64(w, tmp);
                add_to_output64(w, ch, tmp, tmp_e, P.min_rmsd, P.num_saved);
                if (tmp_e < best_e) best_e = tmp_e;
            }
        }
    }
    for (int i = w.lane; i < 625; i += 32) ch.mt[i] = w.mt[i];
    if (w.lane == 0) *ch.evals = w.evals;
}

// non_cache::within
__device__ bool within64(W64& w, double margin) {
    const DModel& m = *w.m;
    const DGeom& G = w.R->g;
    bool ok = true;
    for (int i = w.lane; i < m.nmov; i += 32) {
        if (is_h(m.type[i])) continue;
        for (int j = 0; j < 3; j++)
            if (w.box || G.gd_n[j] > 0) {
                const double c = w.s[w.L.coords + 3 * i + j];
                const double lo = w.box ? w.box[j] : G.gd_begin[j], hi = w.box ? w.box[3 + j] : G.gd_end[j];
                if (c < lo - margin || c > hi + margin) ok = false;
            }
    }
    return __all_sync(kFull, ok);
}

// refine_structure for one pose per block
__global__ void __launch_bounds__(32) k_refine64(const DModel* models, DTables T, const DReceptor* R,
                                                 const int* pose_model, int nposes, double* confs, int conf_stride,
                                                 double c0, double c1, double c2, int maxiters, const int* pose_maxiters,
                                                 const double* pose_box, int accurate, int early, double* out_e,
                                                 double* out_coords, int coord_stride, int* err) {
    const int k = blockIdx.x;
    if (k >= nposes) return;
    const DModel* mp = models + pose_model[k];
    W64 w;
    init_ws64(w, mp, &T, R, err);
    const DModel& m = *mp;
    double* x = w.s + w.L.x_tmp;
    vcopy(w, x, confs + (size_t)k * conf_stride, m.conf_size);
    if (pose_maxiters) maxiters = pose_maxiters[k];  // per-ligand iteration limit
    if (pose_box) w.box = pose_box + 6 * (size_t)k;  // the pose's own box
    double slope = 10;
    double e = 0;
    for (int p = 0; p < 5; p++) {
        const EvalMode em{{c0, c1, c2}, slope, true};
        e = bfgs64(w, x, maxiters, accurate, early, em);
        set_conf64(w, x);
        if (within64(w, 0.0001)) break;
        slope *= 10;
    }
    if (!within64(w, 0.0001)) e = kMaxFl;
    if (w.lane == 0) out_e[k] = e;
    for (int i = w.lane; i < m.conf_size; i += 32) confs[(size_t)k * conf_stride + i] = x[i];
    if (out_coords)
        for (int a = w.lane; a < m.nheavy; a += 32)
            st3(out_coords + ((size_t)k * coord_stride + a) * 3, ld3(w.s + w.L.coords + 3 * m.heavy[a]));
}

// Final rescoring (finish_docking, main.cpp:257-282): per pose, model::eval on
// the direct receptor sum (model.cpp:938-967 with non_cache::eval) and
// model::eval_intramolecular (model.cpp:1027-1079), both on the fast table,
// plus the heavy-atom coordinates of the pose.
__global__ void __launch_bounds__(32) k_score64(const DModel* models, DTables T, const DReceptor* R,
                                                const int* pose_model, int n, const double* confs, int conf_stride,
                                                double v0, double v1, double v2, double slope, double* out_e,
                                                double* out_intra, double* out_coords, int coord_stride, int* err) {
    const int k = blockIdx.x;
    if (k >= n) return;
    W64 w;
    init_ws64(w, models + pose_model[k], &T, R, err);
    const DModel& m = *w.m;
    double* x = w.s + w.L.x_tmp;
    vcopy(w, x, confs + (size_t)k * conf_stride, m.conf_size);
    const double v[3] = {v0, v1, v2};
    set_conf64(w, x);
    direct_energy64(w, v[1], slope);
    pairs_energy64(w, v);
    __syncwarp();
    const double e = energy64(w);
    const double intra = intramolecular64(w, v);
    if (w.lane == 0) {
        out_e[k] = e;
        out_intra[k] = intra;
    }
    if (out_coords)
        for (int a = w.lane; a < m.nheavy; a += 32)
            st3(out_coords + ((size_t)k * coord_stride + a) * 3, ld3(w.s + w.L.coords + 3 * m.heavy[a]));
}

// ---- host launchers -------------------------------------------------------------------------
size_t ws64_bytes(const DModel& hm) {
    return (size_t)ws64_layout(hm.natoms, hm.nframes, hm.npairs, hm.conf_size, hm.dof).total * sizeof(double);
}

static cudaError_t prep(const void* fn, size_t smem) {
    if (smem > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaSuccess;
}

cudaError_t launch_eval64(const DModel* dm, size_t smem, const DTables& T, const DReceptor* R, int n, const double* confs,
                          const double v[3], double slope, int direct, double* e, double* g, double* coords, int* err,
                          cudaStream_t s) {
    cudaError_t rc = prep((const void*)k_eval64, smem);
    if (rc != cudaSuccess) return rc;
    k_eval64<<<n, 32, smem, s>>>(dm, T, R, n, confs, v[0], v[1], v[2], slope, direct, e, g, coords, err);
    return cudaGetLastError();
}

cudaError_t launch_bfgs64(const DModel* dm, size_t smem, const DTables& T, const DReceptor* R, int n, double* confs,
                          const double v[3], double slope, int maxiters, int accurate, int early, double* e, int* err,
                          cudaStream_t s) {
    cudaError_t rc = prep((const void*)k_bfgs64, smem);
    if (rc != cudaSuccess) return rc;
    k_bfgs64<<<n, 32, smem, s>>>(dm, T, R, n, confs, v[0], v[1], v[2], slope, maxiters, accurate, early, e, err);
    return cudaGetLastError();
}

cudaError_t launch_mc64(const DModel* dms, size_t smem, const DTables& T, const DReceptor* R, const Chain64* chains,
                        int n, const MCParams64& P, bool visited, int* err, cudaStream_t s) {
    const void* fn = visited ? (const void*)k_mc64<true> : (const void*)k_mc64<false>;
    cudaError_t rc = prep(fn, smem);
    if (rc != cudaSuccess) return rc;
    if (visited) k_mc64<true><<<n, 32, smem, s>>>(dms, T, R, chains, n, P, err);
    else k_mc64<false><<<n, 32, smem, s>>>(dms, T, R, chains, n, P, err);
    return cudaGetLastError();
}

cudaError_t launch_refine64(const DModel* dms, size_t smem, const DTables& T, const DReceptor* R, const int* pose_model,
                            int n, double* confs, int conf_stride, const double cap[3], int maxiters,
                            const int* pose_maxiters, const double* pose_box, int accurate, int early, double* e,
                            double* coords, int coord_stride, int* err, cudaStream_t s) {
    cudaError_t rc = prep((const void*)k_refine64, smem);
    if (rc != cudaSuccess) return rc;
    k_refine64<<<n, 32, smem, s>>>(dms, T, R, pose_model, n, confs, conf_stride, cap[0], cap[1], cap[2], maxiters,
                                   pose_maxiters, pose_box, accurate, early, e, coords, coord_stride, err);
    return cudaGetLastError();
}

cudaError_t launch_score64(const DModel* dms, size_t smem, const DTables& T, const DReceptor* R, const int* pose_model,
                           int n, const double* confs, int conf_stride, const double v[3], double slope, double* e,
                           double* intra, double* coords, int coord_stride, int* err, cudaStream_t s) {
    cudaError_t rc = prep((const void*)k_score64, smem);
    if (rc != cudaSuccess) return rc;
    k_score64<<<n, 32, smem, s>>>(dms, T, R, pose_model, n, confs, conf_stride, v[0], v[1], v[2], slope, e, intra,
                                  coords, coord_stride, err);
    return cudaGetLastError();
}

}  // namespace sg
