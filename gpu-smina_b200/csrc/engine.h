// Engine state behind the C ABI.
#pragma once
#include <new>
#include <stdexcept>
#include <string>
#include <cstdint>
#include <vector>
#include "sg_dev.cuh"

namespace sg {

struct EngineError : std::runtime_error {
    int code;
    EngineError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);

inline void require(bool ok, const std::string& msg) {
    if (!ok) throw EngineError(SG_ERR_ARG, msg);
}

// owning device allocation
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    void reset();
    void alloc(size_t n);
    void upload(const void* src, size_t n, cudaStream_t s);
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

DGeom make_geom(const sg_grid_dims& gd);

// one resident receptor with its box, cell lists and maps
struct RecState {
    bool set = false;
    sg_grid_dims gd{};
    DGeom geom{};
    int natoms = 0;
    DevBuf xyz, type, charge, pop_start, pop_atoms, full_start, full_atoms;
    DevBuf map64[kNumTypes], cmap64[kNumTypes], map32[kNumTypes], cmap32[kNumTypes], map16[kNumTypes];
    bool built[kNumTypes] = {};
    DevBuf ugrid;  // user grid values, or empty
    DGeom ug{};
    double ug_slope = 1e6;
    DevBuf dhdr;  // device copy of the DReceptor header
    DReceptor hdr{};
    void clear_maps() {
        for (int t = 0; t < kNumTypes; t++) {
            map64[t].reset(); cmap64[t].reset(); map32[t].reset(); cmap32[t].reset(); map16[t].reset();
            built[t] = false;
        }
    }
    size_t map_bytes() const {
        size_t b = 0;
        for (int t = 0; t < kNumTypes; t++)
            b += map64[t].bytes + cmap64[t].bytes + map32[t].bytes + cmap32[t].bytes + map16[t].bytes;
        return b;
    }
};

// a batch of models packed for the device
struct PackedModels {
    std::vector<DModel> host;  // host copies with device pointers
    DevBuf ints, dbls, flts, dmodels;
    size_t max_ws64 = 0;
    int max_conf = 0, max_dof = 0, max_heavy = 0, max_atoms = 0, max_pairs = 0, max_frames = 0;
};

}  // namespace sg

struct sg_engine {
    int device = 0;
    int precision = 0;
    int num_sms = 148;
    int max_smem = 227 * 1024;
    cudaStream_t stream = nullptr;
    std::string err;
    bool has_tables = false;
    sg::DevBuf tab_smooth, tab_fast, tab32;
    int force_wpb = 0, last_wpb = 0, last_blocks = 0;
    int tpc = 32;        // threads per chain of the batched search: 32, 64, 128, or 0 (by the batch's size)
    int last_team = 1;   // warps per chain of the last batched search
    bool es_on = false;   // early stop of the batched search (--fast; sg_set_early_stop)
    sg_early_stop es{};
    double last_mc_ms = 0, last_refine_ms = 0;
    uint64_t last_evals = 0, last_grid_hits = 0, last_pair_hits = 0, last_h2d = 0, last_d2h = 0;
    sg::DTables tables{};
    sg::RecState rec[SG_MAX_RECEPTORS];
    sg::DevBuf d_err;
    ~sg_engine();
    void check_device_errors();
};

namespace sg {

// Runs f() on the engine's device and turns exceptions into status codes
// (the message goes to sg_last_error).
template <typename F>
int guarded(sg_engine* e, F f) {
    try {
        if (!e) return SG_ERR_ARG;
        cuda_check(cudaSetDevice(e->device), "cudaSetDevice");
        f();
        return SG_OK;
    } catch (EngineError& x) {
        e->err = x.what();
        return x.code;
    } catch (std::bad_alloc&) {
        e->err = "host allocation failed";
        return SG_ERR_NOMEM;
    } catch (std::exception& x) {
        e->err = x.what();
        return SG_ERR_ARG;
    }
}

// ---- launchers defined in the kernel files ---------------------------------------------------
cudaError_t launch_cell_lists(int, const double*, const int*, const DGeom&, double, const double*, const double*, int*,
                              const int*, int*, int, cudaStream_t);
cudaError_t launch_grid_map64(const DGeom&, int, const double*, const int*, const double*, const int*, const int*,
                              const DTables&, const int*, int, double**, double**, const double* ugrid,
                              const DGeom& ug, double ug_slope, cudaStream_t);
cudaError_t launch_grid_pack(const DGeom&, const double*, float4*, uint4*, cudaStream_t);
size_t ws64_bytes(const DModel& hm);
cudaError_t launch_eval64(const DModel*, size_t, const DTables&, const DReceptor*, int, const double*, const double[3],
                          double, int, double*, double*, double*, int*, cudaStream_t);
cudaError_t launch_bfgs64(const DModel*, size_t, const DTables&, const DReceptor*, int, double*, const double[3], double,
                          int, int, int, double*, int*, cudaStream_t);
cudaError_t launch_mc64(const DModel*, size_t, const DTables&, const DReceptor*, const Chain64*, int,
                        const MCParams64&, bool visited, int*, cudaStream_t);
cudaError_t launch_score64(const DModel* dms, size_t smem, const DTables& T, const DReceptor* R, const int* pose_model,
                           int n, const double* confs, int conf_stride, const double v[3], double slope, double* e,
                           double* intra, double* coords, int coord_stride, int* err, cudaStream_t s);
cudaError_t launch_refine64(const DModel*, size_t, const DTables&, const DReceptor*, const int*, int, double*, int,
                            const double[3], int, const int* pose_maxiters, const double* pose_box, int, int, double*,
                            double*, int, int*, cudaStream_t);
size_t ws32_bytes(const DModel& hm);
int mc32_occupancy(int team, int wpb, size_t smem);
cudaError_t launch_mc32_feed(const DTables32& T, const FeedItem32* ring, unsigned cap, FeedCtrl32* ctrl,
                             long long idle_ns, int blocks, int wpb, size_t smem, cudaStream_t s);
cudaError_t mc32_feed_reserve_smem(size_t smem);
cudaError_t mc32_feed_occupancy(int wpb, size_t smem, int* blocks);
cudaError_t mc32_feed_max_dynamic_smem(size_t optin, size_t* out);
cudaError_t mc32_reserve_smem(size_t smem);
cudaError_t mc32_max_dynamic_smem(size_t optin, size_t* out);
cudaError_t launch_mc32_fixed(const DModel*, const DTables32&, const DMaps32&, const DMaps32* maps_tab, const Chain32*,
                              const Item32*, int nitems, const MCParams32&, unsigned* queue, int blocks, int wpb,
                              size_t stage_stride, size_t ws_stride, size_t smem_fixed, cudaStream_t s);
cudaError_t launch_mc32(const DModel*, const DTables32&, const DMaps32&, const DMaps32* maps_tab, const Chain32*,
                        const Item32*, int nitems, const MCParams32&, unsigned*, int blocks, int wpb,
                        size_t stage_stride, size_t ws_stride, int team, cudaStream_t);
cudaError_t launch_eval32(const DModel*, size_t stage, size_t ws, const DTables32&, const DMaps32&, int, const double*,
                          const double[3], double, double*, double*, double*, int team, cudaStream_t);
cudaError_t gather_probe(size_t working_set, int bytes_per_lookup, int num_sms, double* gbs, cudaStream_t s);
cudaError_t launch_bfgs32(const DModel*, size_t stage, size_t ws, const DTables32&, const DMaps32&, int, double*,
                          const double v[3], double slope, int maxiters, int accurate, int early, double* e,
                          int team, cudaStream_t);

// FP32 views of the engine's tables and of a receptor's packed maps
DTables32 tables32(const sg_engine* e);
DMaps32 maps32(const sg_engine* e, const RecState& r);
void pack_models(sg_engine* e, const sg_model_desc* models, int nmodels, PackedModels& out);
struct ModelImage {
    std::vector<char> bytes;   // pools then descriptors, ready to copy to the device
    size_t dmodel_off = 0;     // byte offset of the descriptor array
    std::vector<DModel> host;  // the descriptors (device addresses)
};
void pack_models_image(const sg_model_desc* models, int nmodels, char* dev_base, ModelImage& img);
RecState& receptor_for(sg_engine* e, int rid);
void ensure_cells(sg_engine* e, RecState& r);
void ensure_maps(sg_engine* e, RecState& r, const int* types, int ntypes);
void ensure_model_maps(sg_engine* e, RecState& r, const PackedModels& pm, const sg_model_desc* models, int nmodels);
void refresh_header(sg_engine* e, RecState& r);
void serve_shutdown(sg_engine* e);  // stops the engine's request loop, if one runs
// chains per block and resident blocks per SM of a k_mc32 launch (honours
// e->force_wpb)
void choose_launch(sg_engine* e, size_t stage_stride, size_t ws_stride, int max_chains, int& wpb, int& occ);
void noalloc_claim(sg_engine* e);  // the no-allocation entry point's set-up, at engine creation
}  // namespace sg
