// Engine state behind the C ABI.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>
#include "sg_dev.cuh"

namespace sg {

struct EngineError : std::runtime_error {
    int code;
    EngineError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);

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
    DevBuf ints, dbls, dmodels;
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
    sg::DevBuf tab_smooth, tab_fast, tab_smooth32;
    sg::DTables tables{};
    sg::RecState rec[SG_MAX_RECEPTORS];
    sg::DevBuf d_err;
    ~sg_engine();
    void check_device_errors();
};

namespace sg {
void pack_models(sg_engine* e, const sg_model_desc* models, int nmodels, PackedModels& out);
RecState& receptor_for(sg_engine* e, int rid);
void ensure_maps(sg_engine* e, RecState& r, const int* types, int ntypes);
void ensure_model_maps(sg_engine* e, RecState& r, const PackedModels& pm, const sg_model_desc* models, int nmodels);
void refresh_header(sg_engine* e, RecState& r);
}  // namespace sg
