// C ABI of the B200 docking engine (include/smina_b200.h): device state,
// input validation, model packing and kernel launches.  Every entry point
// returns a status code; no exception crosses the ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include "engine.h"

namespace sg {

void DevBuf::reset() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}
void DevBuf::alloc(size_t n) {
    reset();
    if (n == 0) n = 16;
    if (cudaMalloc(&p, n) != cudaSuccess) {
        p = nullptr;
        throw EngineError(SG_ERR_NOMEM, "device allocation of " + std::to_string(n) + " bytes failed");
    }
    bytes = n;
}
void DevBuf::upload(const void* src, size_t n, cudaStream_t s) {
    alloc(n);
    if (n) cuda_check(cudaMemcpyAsync(p, src, n, cudaMemcpyHostToDevice, s), "upload");
}

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        // a failed call that does not poison the context still stays the
        // thread's last error, which the next launch's check would report
        // again; clear it
        cudaGetLastError();
        throw EngineError(SG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

DGeom make_geom(const sg_grid_dims& gd) {
    DGeom g;
    for (int i = 0; i < 3; i++) {
        g.dim[i] = gd.n[i] + 1;
        g.init[i] = gd.begin[i];
        const double range = gd.end[i] - gd.begin[i];
        g.dim_fl_minus_1[i] = g.dim[i] - 1.0;
        g.factor[i] = g.dim_fl_minus_1[i] / range;
        g.factor_inv[i] = 1 / g.factor[i];
        g.gd_begin[i] = gd.begin[i];
        g.gd_end[i] = gd.end[i];
        g.gd_n[i] = gd.n[i];
        g.cell_off[i] = (int)std::floor(gd.begin[i] / 3.0);
        g.cell_dim[i] = (int)std::ceil(gd.end[i] / 3.0) - g.cell_off[i] + 1;
    }
    return g;
}

}  // namespace sg

using namespace sg;

// ---- engine -----------------------------------------------------------------------------------
sg_engine::~sg_engine() {
    if (stream) cudaStreamDestroy(stream);
}

// Reads the device error word, clears it, and turns it into a status.
void sg_engine::check_device_errors() {
    int h = 0;
    cuda_check(cudaMemcpyAsync(&h, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "error word");
    cuda_check(cudaStreamSynchronize(stream), "kernel");
    if (h != kDevOk) {
        const int zero = 0;
        cuda_check(cudaMemcpy(d_err.p, &zero, sizeof(int), cudaMemcpyHostToDevice), "clear error word");
        if (h == kDevOverlap) throw EngineError(SG_ERR_OVERLAP, "Ligand atom exactly overlaps receptor atom.");
        throw EngineError(SG_ERR_ARG, "device reported an out-of-range access (error " + std::to_string(h) + ")");
    }
}

extern "C" {

int sg_create(int device, int precision, sg_engine** out) {
    if (!out) return SG_ERR_ARG;
    *out = nullptr;
    if (precision < SG_PREC_FP64 || precision > SG_PREC_FP32_H16) return SG_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return SG_ERR_CUDA;
    std::unique_ptr<sg_engine> e(new sg_engine());
    e->device = device;
    e->precision = precision;
    int rc = guarded(e.get(), [&] {
        cuda_check(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "stream");
        e->d_err.alloc(sizeof(int));
        cuda_check(cudaMemsetAsync(e->d_err.p, 0, sizeof(int), e->stream), "memset");
        cudaDeviceProp prop;
        cuda_check(cudaGetDeviceProperties(&prop, device), "device properties");
        e->num_sms = prop.multiProcessorCount;
        e->max_smem = (int)prop.sharedMemPerBlockOptin;
        if (precision != SG_PREC_FP64) noalloc_claim(e.get());
    });
    if (rc != SG_OK) return rc;
    *out = e.release();
    return SG_OK;
}

void sg_destroy(sg_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    serve_shutdown(e);
    cudaStreamSynchronize(e->stream);
    delete e;
}

const char* sg_last_error(const sg_engine* e) { return e ? e->err.c_str() : "no engine"; }
int sg_precision(const sg_engine* e) { return e ? e->precision : -1; }

int sg_device_info(const sg_engine* e, int* device, int* num_sms, int* smem_optin) {
    if (!e) return SG_ERR_ARG;
    if (device) *device = e->device;
    if (num_sms) *num_sms = e->num_sms;
    if (smem_optin) *smem_optin = e->max_smem;
    return SG_OK;
}

int sg_set_tables(sg_engine* e, const sg_tables_desc* t) {
    return guarded(e, [&] {
        require(t && t->smooth && t->fast, "tables: null pointers");
        require(t->num_types == SG_NUM_TYPES, "tables: num_types must be 27");
        require(t->num_components == 1 || t->num_components == 4, "tables: num_components must be 1 or 4");
        require(t->factor > 0 && t->cutoff_sqr > 0, "tables: factor and cutoff must be positive");
        require(t->n >= (int)(size_t)(t->factor * t->cutoff_sqr) + 3 && t->n < (1 << 24), "tables: n too small");
        const size_t np = kNumTypePairs;
        e->tab_smooth.upload(t->smooth, np * t->n * t->num_components * 2 * sizeof(double), e->stream);
        e->tab_fast.upload(t->fast, np * t->n * t->num_components * sizeof(double), e->stream);
        // (e_i, dor_i, e_i+1, dor_i+1) per component: one 16 B load per lookup
        {
            const int nc = t->num_components, n = t->n;
            std::vector<float> t4(np * n * nc * 4, 0.f);
            for (size_t pr = 0; pr < np; pr++)
                for (int i = 0; i < n; i++)
                    for (int c = 0; c < nc; c++) {
                        const double* a = t->smooth + ((pr * n + i) * nc + c) * 2;
                        float* o = &t4[((pr * n + i) * nc + c) * 4];
                        o[0] = (float)a[0];
                        o[1] = (float)a[1];
                        if (i + 1 < n) { o[2] = (float)a[nc * 2]; o[3] = (float)a[nc * 2 + 1]; }
                    }
            e->tab32.upload(t4.data(), t4.size() * sizeof(float), e->stream);
        }
        e->tables.nc = t->num_components;
        e->tables.n = t->n;
        e->tables.factor = t->factor;
        e->tables.cutoff_sqr = t->cutoff_sqr;
        e->tables.smooth = (const double*)e->tab_smooth.p;
        e->tables.fast = (const double*)e->tab_fast.p;
        e->has_tables = true;
        for (auto& r : e->rec) r.clear_maps();  // maps depend on the tables
        cuda_check(cudaStreamSynchronize(e->stream), "tables");
    });
}

}  // extern "C"

// ---- receptors and grid maps ----------------------------------------------------------------------
namespace sg {

RecState& receptor_for(sg_engine* e, int rid) {
    require(rid >= 0 && rid < SG_MAX_RECEPTORS, "receptor id out of range");
    require(e->rec[rid].set, "receptor " + std::to_string(rid) + " has not been set");
    return e->rec[rid];
}

void refresh_header(sg_engine* e, RecState& r) {
    DReceptor& h = r.hdr;
    h.natoms = r.natoms;
    h.xyz = r.xyz.as<double>();
    h.type = r.type.as<int>();
    h.charge = r.charge.as<double>();
    h.pop_start = r.pop_start.as<int>();
    h.pop_atoms = r.pop_atoms.as<int>();
    h.full_start = r.full_start.as<int>();
    h.full_atoms = r.full_atoms.as<int>();
    h.g = r.geom;
    for (int t = 0; t < kNumTypes; t++) {
        h.map[t] = r.map64[t].as<double>();
        h.cmap[t] = r.cmap64[t].as<double>();
        h.map32[t] = r.map32[t].as<float4>();
        h.cmap32[t] = r.cmap32[t].as<float4>();
        h.map16[t] = r.map16[t].as<uint4>();
    }
    h.ugrid = r.ugrid.as<double>();
    h.ug = r.ug;
    if (!r.dhdr.p) r.dhdr.alloc(sizeof(DReceptor));
    cuda_check(cudaMemcpyAsync(r.dhdr.p, &h, sizeof(DReceptor), cudaMemcpyHostToDevice, e->stream), "receptor header");
    cuda_check(cudaStreamSynchronize(e->stream), "receptor header");
}

// build one family of cell lists (CSR) on the device
static void build_cells(sg_engine* e, RecState& r, const std::vector<double>& lo, const std::vector<double>& hi,
                        DevBuf& start, DevBuf& atoms) {
    const DGeom& g = r.geom;
    const int ncells = g.cell_dim[0] * g.cell_dim[1] * g.cell_dim[2];
    DevBuf dlo, dhi, dcount;
    dlo.upload(lo.data(), lo.size() * sizeof(double), e->stream);
    dhi.upload(hi.data(), hi.size() * sizeof(double), e->stream);
    dcount.alloc(ncells * sizeof(int));
    cuda_check(launch_cell_lists(r.natoms, r.xyz.as<double>(), r.type.as<int>(), g, e->tables.cutoff_sqr,
                                 dlo.as<double>(), dhi.as<double>(), dcount.as<int>(), nullptr, nullptr, 0, e->stream),
               "cell count");
    std::vector<int> cnt(ncells), st(ncells + 1, 0);
    cuda_check(cudaMemcpyAsync(cnt.data(), dcount.p, ncells * sizeof(int), cudaMemcpyDeviceToHost, e->stream), "counts");
    cuda_check(cudaStreamSynchronize(e->stream), "cell count");
    for (int c = 0; c < ncells; c++) st[c + 1] = st[c] + cnt[c];
    start.upload(st.data(), st.size() * sizeof(int), e->stream);
    atoms.alloc(std::max(1, st[ncells]) * sizeof(int));
    cuda_check(launch_cell_lists(r.natoms, r.xyz.as<double>(), r.type.as<int>(), g, e->tables.cutoff_sqr,
                                 dlo.as<double>(), dhi.as<double>(), nullptr, start.as<int>(), atoms.as<int>(), 1,
                                 e->stream),
               "cell fill");
    cuda_check(cudaStreamSynchronize(e->stream), "cell fill");
}

// Brick of every cell along each axis.  Populate: the first grid point of
// the cell in loop order (floor/ceil of its coordinate, flat when it lies on
// a face); direct sum: the full [3c, 3c + 3) brick.
static void cell_bricks(const DGeom& g, bool first_query, std::vector<double>& lo, std::vector<double>& hi) {
    lo.clear();
    hi.clear();
    const double nan = std::nan("");
    for (int d = 0; d < 3; d++) {
        std::vector<double> l(g.cell_dim[d], nan), h(g.cell_dim[d], nan);
        if (first_query) {
            for (int x = 0; x < g.dim[d]; x++) {
                const double c = g.init[d] + g.factor_inv[d] * x;
                const int cell = (int)std::floor(c / 3.0) - g.cell_off[d];
                if (cell < 0 || cell >= g.cell_dim[d] || l[cell] == l[cell]) continue;
                l[cell] = std::floor(c / 3.0) * 3.0;
                h[cell] = std::ceil(c / 3.0) * 3.0;
            }
        } else {
            for (int c = 0; c < g.cell_dim[d]; c++) {
                l[c] = (double)(c + g.cell_off[d]) * 3.0;
                h[c] = l[c] + 3.0;
            }
        }
        lo.insert(lo.end(), l.begin(), l.end());
        hi.insert(hi.end(), h.begin(), h.end());
    }
}

// the receptor's 3 A cell lists (first-query bricks for the maps, full
// bricks for the direct sum), built once
void ensure_cells(sg_engine* e, RecState& r) {
    if (r.pop_start.p) return;
    std::vector<double> lo, hi;
    cell_bricks(r.geom, true, lo, hi);
    build_cells(e, r, lo, hi, r.pop_start, r.pop_atoms);
    cell_bricks(r.geom, false, lo, hi);
    build_cells(e, r, lo, hi, r.full_start, r.full_atoms);
    refresh_header(e, r);
}

void ensure_maps(sg_engine* e, RecState& r, const int* types, int ntypes) {
    require(e->has_tables, "no tables set");
    std::vector<int> need;
    for (int k = 0; k < ntypes; k++) {
        const int t = types[k];
        require(t >= 0 && t < kNumTypes, "grid type out of range");
        if (!r.built[t] && std::find(need.begin(), need.end(), t) == need.end()) need.push_back(t);
    }
    if (need.empty()) return;
    ensure_cells(e, r);
    const size_t npts = (size_t)r.geom.dim[0] * r.geom.dim[1] * r.geom.dim[2];
    const bool charged = e->tables.nc > 1;
    std::vector<double*> maps, cmaps;
    for (int t : need) {
        r.map64[t].alloc(npts * sizeof(double));
        maps.push_back(r.map64[t].as<double>());
        if (charged) {
            r.cmap64[t].alloc(npts * sizeof(double));
            cmaps.push_back(r.cmap64[t].as<double>());
        } else {
            cmaps.push_back(nullptr);
        }
    }
    DevBuf dtypes, dmaps, dcmaps;
    dtypes.upload(need.data(), need.size() * sizeof(int), e->stream);
    dmaps.upload(maps.data(), maps.size() * sizeof(double*), e->stream);
    dcmaps.upload(cmaps.data(), cmaps.size() * sizeof(double*), e->stream);
    cuda_check(launch_grid_map64(r.geom, r.natoms, r.xyz.as<double>(), r.type.as<int>(), r.charge.as<double>(),
                                 r.pop_start.as<int>(), r.pop_atoms.as<int>(), e->tables, dtypes.as<int>(), (int)need.size(),
                                 dmaps.as<double*>(), dcmaps.as<double*>(), r.ugrid.as<double>(), r.ug, r.ug_slope,
                                 e->stream),
               "grid maps");
    if (e->precision != SG_PREC_FP64) {
        const size_t ncells = (size_t)(r.geom.dim[0] - 1) * (r.geom.dim[1] - 1) * (r.geom.dim[2] - 1);
        for (int t : need) {
            r.map32[t].alloc(ncells * 2 * sizeof(float4));
            if (e->precision == SG_PREC_FP32_H16) r.map16[t].alloc(ncells * sizeof(uint4));
            cuda_check(launch_grid_pack(r.geom, r.map64[t].as<double>(), r.map32[t].as<float4>(), r.map16[t].as<uint4>(),
                                        e->stream),
                       "pack maps");
            if (charged) {
                r.cmap32[t].alloc(ncells * 2 * sizeof(float4));
                cuda_check(launch_grid_pack(r.geom, r.cmap64[t].as<double>(), r.cmap32[t].as<float4>(), nullptr, e->stream),
                           "pack charge maps");
            }
        }
    }
    cuda_check(cudaStreamSynchronize(e->stream), "grid maps");
    for (int t : need) r.built[t] = true;
    refresh_header(e, r);
}

}  // namespace sg

extern "C" {

int sg_set_receptor(sg_engine* e, int rid, const sg_receptor_desc* r, const sg_grid_dims* gd) {
    return guarded(e, [&] {
        require(rid >= 0 && rid < SG_MAX_RECEPTORS, "receptor id out of range");
        require(r && gd && r->num_atoms >= 0, "receptor: bad arguments");
        require(r->num_atoms == 0 || (r->coords && r->type && r->charge), "receptor: null arrays");
        require(e->has_tables, "set tables before the receptor");
        for (int i = 0; i < 3; i++) {
            require(gd->n[i] >= 1 && gd->n[i] <= 4096, "box: n must be in [1, 4096]");
            require(gd->end[i] > gd->begin[i], "box: end must exceed begin");
        }
        for (int i = 0; i < r->num_atoms; i++) require(std::isfinite(r->coords[3 * i]) && std::isfinite(r->coords[3 * i + 1]) &&
                                                           std::isfinite(r->coords[3 * i + 2]), "receptor: non-finite coordinate");
        RecState& s = e->rec[rid];
        s.clear_maps();
        s.pop_start.reset(); s.pop_atoms.reset(); s.full_start.reset(); s.full_atoms.reset();
        s.ugrid.reset();  // a new receptor starts without a user grid
        s.ug = DGeom{};
        s.gd = *gd;
        s.geom = make_geom(*gd);
        s.natoms = r->num_atoms;
        std::vector<int> types(r->type, r->type + r->num_atoms);
        for (int& t : types) if (t < 0 || t > kNumTypes) t = kNumTypes;
        s.xyz.upload(r->coords, sizeof(double) * 3 * std::max(1, r->num_atoms), e->stream);
        s.type.upload(types.data(), sizeof(int) * std::max<size_t>(1, types.size()), e->stream);
        s.charge.upload(r->charge, sizeof(double) * std::max(1, r->num_atoms), e->stream);
        s.set = true;
        std::vector<double> lo, hi;
        cell_bricks(s.geom, true, lo, hi);
        build_cells(e, s, lo, hi, s.pop_start, s.pop_atoms);
        cell_bricks(s.geom, false, lo, hi);
        build_cells(e, s, lo, hi, s.full_start, s.full_atoms);
        refresh_header(e, s);
    });
}

int sg_build_grids(sg_engine* e, int rid, const int* types, int ntypes) {
    return guarded(e, [&] {
        require(ntypes >= 0 && (ntypes == 0 || types), "build_grids: bad type list");
        RecState& r = receptor_for(e, rid);
        ensure_maps(e, r, types, ntypes);
    });
}

int sg_get_grid(sg_engine* e, int rid, int type, double* data, double* chargedata) {
    return guarded(e, [&] {
        RecState& r = receptor_for(e, rid);
        require(type >= 0 && type < kNumTypes && r.built[type], "grid map not built");
        require(data != nullptr, "null output");
        cuda_check(cudaMemcpy(data, r.map64[type].p, r.map64[type].bytes, cudaMemcpyDeviceToHost), "get grid");
        if (chargedata && r.cmap64[type].p)
            cuda_check(cudaMemcpy(chargedata, r.cmap64[type].p, r.cmap64[type].bytes, cudaMemcpyDeviceToHost), "get grid");
    });
}

int sg_set_user_grid(sg_engine* e, int rid, const sg_grid_dims* gd, const double* data, double cache_slope) {
    return guarded(e, [&] {
        RecState& r = receptor_for(e, rid);
        if (gd && data) {
            for (int i = 0; i < 3; i++) {
                require(gd->n[i] >= 1 && gd->n[i] <= 4096, "user grid: n must be in [1, 4096]");
                require(gd->end[i] > gd->begin[i], "user grid: end must exceed begin");
            }
            require(std::isfinite(cache_slope), "user grid: non-finite slope");
            const size_t n = (size_t)(gd->n[0] + 1) * (gd->n[1] + 1) * (gd->n[2] + 1);
            for (size_t k = 0; k < n; k++) require(std::isfinite(data[k]), "user grid: non-finite value");
            r.ugrid.upload(data, n * sizeof(double), e->stream);
            r.ug = make_geom(*gd);
            r.ug_slope = cache_slope;
        } else {
            r.ugrid.reset();
            r.ug = DGeom{};
        }
        r.clear_maps();
        refresh_header(e, r);
    });
}

int sg_drop_receptor(sg_engine* e, int rid) {
    return guarded(e, [&] {
        require(rid >= 0 && rid < SG_MAX_RECEPTORS, "receptor id out of range");
        RecState& s = e->rec[rid];
        s.clear_maps();
        s.pop_start.reset(); s.pop_atoms.reset(); s.full_start.reset(); s.full_atoms.reset();
        s.xyz.reset(); s.type.reset(); s.charge.reset(); s.dhdr.reset(); s.ugrid.reset();
        s.set = false;
    });
}

}  // extern "C"

// ---- models -------------------------------------------------------------------------------------------
namespace sg {

// Validates one model descriptor on the host so that no device index can
// leave its array, then appends its packed arrays.
// Mixed-precision pair schedule: chunks of 32 slots in which no atom is
// the first atom of two pairs and none is the second atom of two pairs, so
// one warp adds a chunk's forces without atomics (first atoms, then second
// atoms).  A pair may be stored either way round: swapping the atoms toggles
// the charge-role bit.  Within each quarter of a chunk (the 8 lanes that one
// 16-byte shared-memory access serves at a time) the first atoms are
// distinct modulo 8 and so are the second atoms, so the per-atom float4
// loads and stores of a quarter hit 8 different bank groups.  pair_tp[k]:
// type-pair index | (1 << 30) when the pair's first type is the larger.
// Returns false (no schedule) for models of more than 255 atoms.
static bool pack_pair_chunks(const sg_model_desc& d, const std::vector<int>& pair_tp, std::vector<uint32_t>& out) {
    const int N = d.num_atoms, P = d.num_pairs;
    out.clear();
    if (N > 255) return false;  // 8-bit atom indices (inflex atoms take part in pairs too)
    struct Chunk {
        std::vector<char> out_used, in_used;
        uint8_t amod[4] = {}, bmod[4] = {};  // bank groups taken per quarter (bit masks)
        uint32_t slot[32];
        int fill[4] = {};
    };
    std::vector<Chunk> chunks;
    for (int k = 0; k < P; k++) {
        const int u = d.pairs[2 * k], v = d.pairs[2 * k + 1];
        require(u >= 0 && v >= 0 && u < N && v < N && u != v, "model: pair atoms must be distinct atoms");
        require((pair_tp[k] & 0x1ff) < (int)kSlotPairMask, "model: type pair index out of range");
        const uint32_t base = ((uint32_t)(pair_tp[k] & 0x1ff) << 16) | ((pair_tp[k] >> 30) & 1 ? kSlotSwap : 0) |
                              (k >= d.num_other_pairs ? kSlotIntra : 0);
        bool placed = false;
        for (size_t c = 0; c < chunks.size() && !placed; c++) {
            Chunk& ch = chunks[c];
            for (int o = 0; o < 2 && !placed; o++) {
                const int a = o ? v : u, b = o ? u : v;
                if (ch.out_used[a] || ch.in_used[b]) continue;
                for (int q = 0; q < 4; q++) {
                    if (ch.fill[q] == 8 || (ch.amod[q] >> (a & 7) & 1) || (ch.bmod[q] >> (b & 7) & 1)) continue;
                    ch.out_used[a] = ch.in_used[b] = 1;
                    ch.amod[q] |= 1 << (a & 7);
                    ch.bmod[q] |= 1 << (b & 7);
                    ch.slot[8 * q + ch.fill[q]++] = (o ? base ^ kSlotSwap : base) | a | (b << 8);
                    placed = true;
                    break;
                }
            }
        }
        if (!placed) {
            chunks.emplace_back();
            Chunk& ch = chunks.back();
            ch.out_used.assign(N, 0);
            ch.in_used.assign(N, 0);
            for (uint32_t& x : ch.slot) x = kSlotEmpty;
            ch.out_used[u] = ch.in_used[v] = 1;
            ch.amod[0] = 1 << (u & 7);
            ch.bmod[0] = 1 << (v & 7);
            ch.slot[ch.fill[0]++] = base | u | (v << 8);
        }
    }
    for (const Chunk& ch : chunks) out.insert(out.end(), ch.slot, ch.slot + 32);
    return true;
}

static void pack_one(const sg_model_desc& d, std::vector<int>& I, std::vector<double>& D, std::vector<float>& Fl,
                     std::vector<size_t>& ioff, std::vector<size_t>& doff, std::vector<size_t>& foff, DModel& hm) {
    const int N = d.num_atoms, M = d.num_movable, F = d.num_frames, P = d.num_pairs;
    require(N > 0 && N <= 4096 && M > 0 && M <= N, "model: atom counts out of range");
    require(F > 0 && F <= 1024 && d.num_ligands >= 0 && d.num_flex >= 0 && d.num_ligands + d.num_flex > 0,
            "model: frame / ligand counts out of range");
    require(d.num_ligands <= 30, "model: at most 30 ligands per model");
    require(P >= 0 && P <= 200000 && d.num_other_pairs >= 0 && d.num_other_pairs <= P, "model: pair counts out of range");
    require(d.conf_size > 0 && d.conf_size <= 4096 && d.dof > 0 && d.dof <= 1024, "model: conf/dof sizes out of range");
    require(d.atom_type && d.atom_charge && d.atom_local && d.atom_lab && d.frame_kind && d.frame_parent &&
                d.frame_begin && d.frame_end && d.frame_conf && d.frame_dof && d.frame_origin && d.frame_axis &&
                d.frame_init_origin && (P == 0 || d.pairs) && (d.num_ligands == 0 || (d.lig_pair_end &&
                d.ligand_atom_begin && d.ligand_atom_end && d.ligand_root)),
            "model: null arrays");
    // frames
    std::vector<int> depth(F, 0), atom_frame(N, -1);
    int nlevels = 1, nlig_roots = 0, nflex_roots = 0;
    for (int f = 0; f < F; f++) {
        const int k = d.frame_kind[f], p = d.frame_parent[f];
        require(k >= 0 && k <= 2, "model: bad frame kind");
        require((k == SG_FRAME_SEGMENT) == (p >= 0), "model: only segments have parents");
        require(p < f, "model: frames must be in depth-first order");
        depth[f] = p < 0 ? 0 : depth[p] + 1;
        nlevels = std::max(nlevels, depth[f] + 1);
        require(d.frame_begin[f] >= 0 && d.frame_begin[f] <= d.frame_end[f] && d.frame_end[f] <= M,
                "model: frame atom range out of range");
        for (int i = d.frame_begin[f]; i < d.frame_end[f]; i++) {
            require(atom_frame[i] < 0, "model: frames overlap");
            atom_frame[i] = f;
        }
        if (k == SG_FRAME_RIGID) {
            require(d.frame_conf[f] >= 0 && d.frame_conf[f] + 7 <= d.conf_size && d.frame_dof[f] >= 0 &&
                        d.frame_dof[f] + 6 <= d.dof, "model: rigid conf/dof offsets out of range");
            nlig_roots++;
        } else {
            require(d.frame_conf[f] >= 0 && d.frame_conf[f] < d.conf_size && d.frame_dof[f] >= 0 && d.frame_dof[f] < d.dof,
                    "model: torsion conf/dof offsets out of range");
            if (k == SG_FRAME_FIRST_SEGMENT) nflex_roots++;
        }
        for (int j = 0; j < 3; j++)
            require(std::isfinite(d.frame_origin[3 * f + j]) && std::isfinite(d.frame_axis[3 * f + j]) &&
                        std::isfinite(d.frame_init_origin[3 * f + j]), "model: non-finite frame data");
    }
    require(nlig_roots == d.num_ligands && nflex_roots == d.num_flex, "model: root counts disagree with ligands/flex");
    for (int i = 0; i < M; i++) require(atom_frame[i] >= 0, "model: a movable atom belongs to no frame");
    for (int i = 0; i < N; i++) {
        require(d.atom_type[i] >= 0 && d.atom_type[i] <= kNumTypes, "model: atom type out of range");
        for (int j = 0; j < 3; j++)
            require(std::isfinite(d.atom_local[3 * i + j]) && std::isfinite(d.atom_lab[3 * i + j]), "model: non-finite atom data");
    }
    for (int l = 0; l < d.num_ligands; l++) {
        require(d.ligand_root[l] >= 0 && d.ligand_root[l] < F && d.frame_kind[d.ligand_root[l]] == SG_FRAME_RIGID,
                "model: ligand root is not a rigid frame");
        require(d.ligand_atom_begin[l] >= 0 && d.ligand_atom_begin[l] <= d.ligand_atom_end[l] && d.ligand_atom_end[l] <= M,
                "model: ligand atom range out of range");
        const int prev = l == 0 ? d.num_other_pairs : d.lig_pair_end[l - 1];
        require(d.lig_pair_end[l] >= prev && d.lig_pair_end[l] <= P, "model: ligand pair ranges out of order");
    }
    require(d.num_ligands == 0 || d.lig_pair_end[d.num_ligands - 1] == P, "model: pairs not covered by ligand ranges");
    if (d.num_ligands == 0) require(d.num_other_pairs == P, "model: pairs not covered");
    // levels, children
    std::vector<int> level_start(nlevels + 1, 0), level_frames;
    for (int lv = 0; lv < nlevels; lv++) {
        level_start[lv] = (int)level_frames.size();
        for (int f = 0; f < F; f++) if (depth[f] == lv) level_frames.push_back(f);
    }
    level_start[nlevels] = (int)level_frames.size();
    std::vector<int> child_start(F + 1, 0), child_list;
    for (int f = 0; f < F; f++) {
        child_start[f] = (int)child_list.size();
        for (int c = f + 1; c < F; c++) if (d.frame_parent[c] == f) child_list.push_back(c);
    }
    child_start[F] = (int)child_list.size();
    // pairs, groups, per-atom ordered pair lists
    std::vector<int> group(P, 0), pair_tp(P, 0);
    for (int k = 0; k < P; k++) {
        const int a = d.pairs[2 * k], b = d.pairs[2 * k + 1];
        require(a >= 0 && a < N && b >= 0 && b < N && a != b, "model: pair atom out of range");
        const int ta = d.atom_type[a], tb = d.atom_type[b];
        require(ta < kNumTypes && tb < kNumTypes, "model: a pair atom has no type");
        pair_tp[k] = (ta <= tb ? tri_index(ta, tb) : tri_index(tb, ta)) | (ta > tb ? (1 << 30) : 0);
        if (k >= d.num_other_pairs)
            for (int l = 0; l < d.num_ligands; l++)
                if (k < d.lig_pair_end[l]) { group[k] = l + 1; break; }
    }
    std::vector<std::vector<int>> lists(M);
    for (int k = 0; k < P; k++) {
        const int a = d.pairs[2 * k], b = d.pairs[2 * k + 1];
        if (a < M) lists[a].push_back(k << 1);
        if (b < M) lists[b].push_back((k << 1) | 1);
    }
    std::vector<int> csr_start(M + 1, 0), csr;
    for (int i = 0; i < M; i++) {
        csr_start[i] = (int)csr.size();
        csr.insert(csr.end(), lists[i].begin(), lists[i].end());
    }
    csr_start[M] = (int)csr.size();
    std::vector<int> heavy;
    for (int i = 0; i < M; i++) if (!is_h(d.atom_type[i])) heavy.push_back(i);
    // conf blocks (ligands, then flexible residues) and their torsions
    std::vector<int> root_of(F);
    for (int f = 0; f < F; f++) root_of[f] = d.frame_parent[f] < 0 ? f : root_of[d.frame_parent[f]];
    std::vector<int> blk_rigid, blk_conf, blk_dof, blk_ntors, tor_conf, tor_dof, tor_frame;
    for (int pass = 0; pass < 2; pass++)
        for (int f = 0; f < F; f++) {
            if (d.frame_parent[f] >= 0) continue;
            const bool rigid = d.frame_kind[f] == SG_FRAME_RIGID;
            if ((pass == 0) != rigid) continue;
            blk_rigid.push_back(rigid);
            blk_conf.push_back(d.frame_conf[f]);
            blk_dof.push_back(d.frame_dof[f]);
            int nt = 0;
            for (int g = 0; g < F; g++)
                if (root_of[g] == f && d.frame_kind[g] != SG_FRAME_RIGID) {
                    const int expect_c = d.frame_conf[f] + (rigid ? 7 : 0) + nt;
                    const int expect_d = d.frame_dof[f] + (rigid ? 6 : 0) + nt;
                    require(d.frame_conf[g] == expect_c && d.frame_dof[g] == expect_d,
                            "model: torsions must follow their block in depth-first order");
                    tor_conf.push_back(d.frame_conf[g]);
                    tor_dof.push_back(d.frame_dof[g]);
                    tor_frame.push_back(g);
                    nt++;
                }
            blk_ntors.push_back(nt);
        }
    // pack
    auto pi = [&](const int* src, size_t n) { ioff.push_back(I.size()); I.insert(I.end(), src, src + n); };
    auto pv = [&](const std::vector<int>& v) { ioff.push_back(I.size()); I.insert(I.end(), v.begin(), v.end()); I.push_back(0); };
    auto pd = [&](const double* src, size_t n) { doff.push_back(D.size()); D.insert(D.end(), src, src + n); };
    ioff.clear();
    doff.clear();
    const size_t i0 = I.size(), d0 = D.size();
    (void)i0; (void)d0;
    pi(d.atom_type, N); pi(d.frame_kind, F); pi(d.frame_parent, F); pi(d.frame_begin, F); pi(d.frame_end, F);
    pi(d.frame_conf, F); pi(d.frame_dof, F);
    pv(atom_frame); pv(level_start); pv(level_frames); pv(child_start); pv(child_list);
    if (I.size() & 1) I.push_back(0);  // pairs are read as int2
    if (P) pi(d.pairs, 2 * (size_t)P); else pv({});
    pv(group); pv(csr_start); pv(csr); pv(heavy);
    std::vector<int> lb(d.ligand_atom_begin, d.ligand_atom_begin + d.num_ligands),
        le(d.ligand_atom_end, d.ligand_atom_end + d.num_ligands), lr(d.ligand_root, d.ligand_root + d.num_ligands),
        lp(d.lig_pair_end, d.lig_pair_end + d.num_ligands);
    pv(lb); pv(le); pv(lr); pv(lp);
    pv(blk_rigid); pv(blk_conf); pv(blk_dof); pv(blk_ntors); pv(tor_conf); pv(tor_dof); pv(tor_frame);
    pv(pair_tp);
    {   // subtree atom ranges: a frame's descendants follow its own atoms
        std::vector<int> sub_end(F);
        for (int f = F - 1; f >= 0; f--) {
            sub_end[f] = d.frame_end[f];
            for (int c = f + 1; c < F; c++)
                if (d.frame_parent[c] == f) sub_end[f] = std::max(sub_end[f], sub_end[c]);
        }
        for (int c = 0; c < F; c++)
            for (int a = d.frame_parent[c]; a >= 0; a = d.frame_parent[a])
                require(d.frame_begin[c] >= d.frame_end[a] && d.frame_end[c] <= sub_end[a],
                        "model: a subtree's atoms must follow its root frame's atoms contiguously");
        pv(sub_end);
    }
    {   // mixed-precision pair schedule (pack_pair_chunks)
        std::vector<uint32_t> slots;
        const bool packable = pack_pair_chunks(d, pair_tp, slots);
        std::vector<int> ps(slots.begin(), slots.end());
        hm.npchunks = packable ? (int)(slots.size() / 32) : -1;
        pv(ps);
    }
    auto pf4 = [&](const double* xyz, const double* w4, size_t n) {
        foff.push_back(Fl.size());
        for (size_t i = 0; i < n; i++) {
            Fl.push_back((float)xyz[3 * i]); Fl.push_back((float)xyz[3 * i + 1]); Fl.push_back((float)xyz[3 * i + 2]);
            Fl.push_back(w4 ? (float)w4[i] : 0.f);
        }
    };
    foff.clear();
    pf4(d.atom_local, d.atom_charge, N); pf4(d.atom_lab, nullptr, N);
    pf4(d.frame_origin, nullptr, F); pf4(d.frame_axis, nullptr, F); pf4(d.frame_init_origin, nullptr, F);
    hm.cost = M + P + 8 * F;
    pd(d.atom_charge, N); pd(d.atom_local, 3 * (size_t)N); pd(d.atom_lab, 3 * (size_t)N);
    pd(d.frame_origin, 3 * (size_t)F); pd(d.frame_axis, 3 * (size_t)F); pd(d.frame_init_origin, 3 * (size_t)F);
    hm.natoms = N; hm.nmov = M; hm.nframes = F; hm.nlig = d.num_ligands; hm.nflex = d.num_flex;
    hm.conf_size = d.conf_size; hm.dof = d.dof; hm.npairs = P; hm.nother = d.num_other_pairs;
    hm.nheavy = (int)heavy.size(); hm.nlevels = nlevels; hm.nblocks = (int)blk_rigid.size();
    hm.ntors = (int)tor_conf.size();
    require(hm.ntors + 6 * d.num_ligands == d.dof, "model: dof disagrees with the torsion count");
}

void pack_models(sg_engine* e, const sg_model_desc* models, int nmodels, PackedModels& out) {
    require(models && nmodels > 0 && nmodels <= (1 << 20), "models: bad array");
    std::vector<int> I;
    std::vector<double> D;
    std::vector<float> Fl;
    std::vector<std::vector<size_t>> ioffs(nmodels), doffs(nmodels), foffs(nmodels);
    out.host.assign(nmodels, DModel{});
    for (int k = 0; k < nmodels; k++) pack_one(models[k], I, D, Fl, ioffs[k], doffs[k], foffs[k], out.host[k]);
    out.ints.upload(I.data(), std::max<size_t>(1, I.size()) * sizeof(int), e->stream);
    out.dbls.upload(D.data(), std::max<size_t>(1, D.size()) * sizeof(double), e->stream);
    out.flts.upload(Fl.data(), std::max<size_t>(4, Fl.size()) * sizeof(float), e->stream);
    const int* ib = out.ints.as<int>();
    const double* db = out.dbls.as<double>();
    const float* fb = out.flts.as<float>();
    out.max_ws64 = 0;
    for (int k = 0; k < nmodels; k++) {
        DModel& h = out.host[k];
        const std::vector<size_t>& io = ioffs[k];
        const std::vector<size_t>& dd = doffs[k];
        int j = 0;
        h.type = ib + io[j++]; h.fkind = ib + io[j++]; h.fparent = ib + io[j++]; h.fbegin = ib + io[j++];
        h.fend = ib + io[j++]; h.fconf = ib + io[j++]; h.fdof = ib + io[j++];
        h.atom_frame = ib + io[j++]; h.level_start = ib + io[j++]; h.level_frames = ib + io[j++];
        h.child_start = ib + io[j++]; h.child_list = ib + io[j++]; h.pairs = ib + io[j++];
        h.pair_group = ib + io[j++]; h.csr_start = ib + io[j++]; h.csr = ib + io[j++]; h.heavy = ib + io[j++];
        h.lig_begin = ib + io[j++]; h.lig_end = ib + io[j++]; h.lig_root = ib + io[j++]; h.lig_pair_end = ib + io[j++];
        h.blk_rigid = ib + io[j++]; h.blk_conf = ib + io[j++]; h.blk_dof = ib + io[j++]; h.blk_ntors = ib + io[j++];
        h.tor_conf = ib + io[j++]; h.tor_dof = ib + io[j++]; h.tor_frame = ib + io[j++];
        h.pair_tp = ib + io[j++];
        h.fsub_end = ib + io[j++];
        h.pslot = h.npchunks >= 0 ? (const uint32_t*)(ib + io[j]) : nullptr;
        j++;
        const std::vector<size_t>& fo = foffs[k];
        h.local32 = (const float4*)(fb + fo[0]); h.lab32 = (const float4*)(fb + fo[1]);
        h.forigin32 = (const float4*)(fb + fo[2]); h.faxis32 = (const float4*)(fb + fo[3]);
        h.finit32 = (const float4*)(fb + fo[4]);
        int q = 0;
        h.charge = db + dd[q++]; h.local = db + dd[q++]; h.lab = db + dd[q++];
        h.forigin = db + dd[q++]; h.faxis = db + dd[q++]; h.finit = db + dd[q++];
        out.max_ws64 = std::max(out.max_ws64, ws64_bytes(h));
        out.max_conf = std::max(out.max_conf, h.conf_size);
        out.max_dof = std::max(out.max_dof, h.dof);
        out.max_heavy = std::max(out.max_heavy, h.nheavy);
        out.max_atoms = std::max(out.max_atoms, h.natoms);
        out.max_pairs = std::max(out.max_pairs, h.npairs);
        out.max_frames = std::max(out.max_frames, h.nframes);
    }
    out.dmodels.upload(out.host.data(), out.host.size() * sizeof(DModel), e->stream);
    cuda_check(cudaStreamSynchronize(e->stream), "model upload");
}

// Host image of the packed models for a caller that places them in device
// memory it already owns: the int, double and float pools and then the
// descriptors, each 16 B aligned, with every descriptor pointer aimed at
// dev_base + its offset in the image.
void pack_models_image(const sg_model_desc* models, int nmodels, char* dev_base, ModelImage& img) {
    require(models && nmodels > 0 && nmodels <= (1 << 20), "models: bad array");
    std::vector<int> I;
    std::vector<double> D;
    std::vector<float> Fl;
    std::vector<std::vector<size_t>> ioffs(nmodels), doffs(nmodels), foffs(nmodels);
    img.host.assign(nmodels, DModel{});
    for (int k = 0; k < nmodels; k++) pack_one(models[k], I, D, Fl, ioffs[k], doffs[k], foffs[k], img.host[k]);
    auto r16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t oi = 0, od = r16(I.size() * sizeof(int)), of = od + r16(D.size() * sizeof(double));
    img.dmodel_off = of + r16(Fl.size() * sizeof(float));
    img.bytes.assign(img.dmodel_off + nmodels * sizeof(DModel), 0);
    std::memcpy(img.bytes.data() + oi, I.data(), I.size() * sizeof(int));
    std::memcpy(img.bytes.data() + od, D.data(), D.size() * sizeof(double));
    std::memcpy(img.bytes.data() + of, Fl.data(), Fl.size() * sizeof(float));
    const int* ib = reinterpret_cast<const int*>(dev_base + oi);
    const double* db = reinterpret_cast<const double*>(dev_base + od);
    const float* fb = reinterpret_cast<const float*>(dev_base + of);
    for (int k = 0; k < nmodels; k++) {
        DModel& h = img.host[k];
        const std::vector<size_t>& io = ioffs[k];
        const std::vector<size_t>& dd = doffs[k];
        const std::vector<size_t>& fo = foffs[k];
        const int** ip[] = {&h.type, &h.fkind, &h.fparent, &h.fbegin, &h.fend, &h.fconf, &h.fdof, &h.atom_frame,
                            &h.level_start, &h.level_frames, &h.child_start, &h.child_list, &h.pairs, &h.pair_group,
                            &h.csr_start, &h.csr, &h.heavy, &h.lig_begin, &h.lig_end, &h.lig_root, &h.lig_pair_end,
                            &h.blk_rigid, &h.blk_conf, &h.blk_dof, &h.blk_ntors, &h.tor_conf, &h.tor_dof,
                            &h.tor_frame, &h.pair_tp, &h.fsub_end};
        size_t j = 0;
        for (const int** q : ip) *q = ib + io[j++];
        h.pslot = h.npchunks >= 0 ? reinterpret_cast<const uint32_t*>(ib + io[j]) : nullptr;
        const float4** fp[] = {&h.local32, &h.lab32, &h.forigin32, &h.faxis32, &h.finit32};
        j = 0;
        for (const float4** q : fp) *q = reinterpret_cast<const float4*>(fb + fo[j++]);
        const double** dp[] = {&h.charge, &h.local, &h.lab, &h.forigin, &h.faxis, &h.finit};
        j = 0;
        for (const double** q : dp) *q = db + dd[j++];
    }
    std::memcpy(img.bytes.data() + img.dmodel_off, img.host.data(), nmodels * sizeof(DModel));
}

void ensure_model_maps(sg_engine* e, RecState& r, const PackedModels& pm, const sg_model_desc* models, int nmodels) {
    std::vector<int> types;
    for (int k = 0; k < nmodels; k++)
        for (int i = 0; i < models[k].num_movable; i++) {
            const int t = models[k].atom_type[i];
            if (t < kNumTypes && !is_h(t)) types.push_back(t);
        }
    (void)pm;
    ensure_maps(e, r, types.data(), (int)types.size());
}

}  // namespace sg

// device buffer that receives results and is copied back
template <typename T>
struct Staged {
    sg::DevBuf d;
    size_t n = 0;
    void make(size_t count, cudaStream_t s, const T* init = nullptr) {
        n = count;
        d.alloc(std::max<size_t>(1, n) * sizeof(T));
        if (init) sg::cuda_check(cudaMemcpyAsync(d.p, init, n * sizeof(T), cudaMemcpyHostToDevice, s), "stage in");
    }
    T* p() { return d.as<T>(); }
    void zero(cudaStream_t s) {  // for outputs with padding the kernel leaves alone
        sg::cuda_check(cudaMemsetAsync(d.p, 0, std::max<size_t>(1, n) * sizeof(T), s), "zero output");
    }
    void fetch(T* host, cudaStream_t s) {
        if (host && n) sg::cuda_check(cudaMemcpyAsync(host, d.p, n * sizeof(T), cudaMemcpyDeviceToHost, s), "stage out");
    }
};

extern "C" {

static int eval_common(sg_engine* e, int rid, const sg_model_desc* m, int nconfs, const double* confs, const double v[3],
                       double slope, double* out_e, double* out_g, double* out_coords, int direct) {
    return guarded(e, [&] {
        require(m && confs && v && out_e && out_g && nconfs > 0 && nconfs <= (1 << 24), "eval: bad arguments");
        require(e->has_tables, "no tables set");
        RecState& r = receptor_for(e, rid);
        PackedModels pm;
        pack_models(e, m, 1, pm);
        if (!direct) ensure_model_maps(e, r, pm, m, 1);
        else ensure_cells(e, r);
        require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
        const DModel& h = pm.host[0];
        Staged<double> dc, de, dg, dx;
        dc.make((size_t)nconfs * h.conf_size, e->stream, confs);
        de.make(nconfs, e->stream);
        dg.make((size_t)nconfs * h.dof, e->stream);
        if (out_coords) dx.make((size_t)nconfs * h.nmov * 3, e->stream);
        if (!direct && e->precision != SG_PREC_FP64) {  // the mixed-precision evaluation
            require(h.npchunks >= 0, "mixed-precision path: at most 255 atoms per model");
            const size_t ws = (ws32_bytes(h) + 15) & ~(size_t)15;
            const size_t stage =
                (size_t)stage32_bytes(h.natoms, h.nframes, h.nheavy, h.npchunks, h.nlig, h.nblocks, h.ntors);
            require(stage + (size_t)std::max(1, e->tpc / 32) * ws <= (size_t)e->max_smem,
                    "model too large for the mixed-precision path's shared memory");
            cuda_check(launch_eval32(pm.dmodels.as<DModel>(), stage, ws, tables32(e), maps32(e, r), nconfs, dc.p(), v, slope,
                                     de.p(), dg.p(), out_coords ? dx.p() : nullptr, std::max(1, e->tpc / 32), e->stream),
                       "eval launch");
            de.fetch(out_e, e->stream);
            dg.fetch(out_g, e->stream);
            if (out_coords) dx.fetch(out_coords, e->stream);
            e->check_device_errors();
            return;
        }
        cuda_check(launch_eval64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(), nconfs, dc.p(), v,
                                 slope, direct, de.p(), dg.p(), out_coords ? dx.p() : nullptr, e->d_err.as<int>(), e->stream),
                   "eval launch");
        de.fetch(out_e, e->stream);
        dg.fetch(out_g, e->stream);
        if (out_coords) dx.fetch(out_coords, e->stream);
        e->check_device_errors();
    });
}

int sg_eval(sg_engine* e, int rid, const sg_model_desc* m, int nconfs, const double* confs, const double v[3],
            double slope, double* out_e, double* out_g, double* out_coords) {
    return eval_common(e, rid, m, nconfs, confs, v, slope, out_e, out_g, out_coords, 0);
}

int sg_eval_direct(sg_engine* e, int rid, const sg_model_desc* m, int nconfs, const double* confs, const double v[3],
                   double slope, double* out_e, double* out_g) {
    return eval_common(e, rid, m, nconfs, confs, v, slope, out_e, out_g, nullptr, 1);
}

int sg_probe_gather(sg_engine* e, uint64_t working_set_bytes, int bytes_per_lookup, double* out_gbs) {
    return guarded(e, [&] {
        require(out_gbs && (bytes_per_lookup == 16 || bytes_per_lookup == 32) && working_set_bytes >= (1u << 20) &&
                    working_set_bytes <= (64ull << 30),
                "probe_gather: bad arguments");
        cuda_check(gather_probe(working_set_bytes, bytes_per_lookup, e->num_sms, out_gbs, e->stream), "gather probe");
    });
}

int sg_bfgs(sg_engine* e, int rid, const sg_model_desc* m, int nconfs, double* confs, const double v[3], double slope,
            int maxiters, int accurate_line, int early_term, double* out_e) {
    return guarded(e, [&] {
        require(m && confs && v && out_e && nconfs > 0 && nconfs <= (1 << 24) && maxiters >= 0, "bfgs: bad arguments");
        RecState& r = receptor_for(e, rid);
        PackedModels pm;
        pack_models(e, m, 1, pm);
        ensure_model_maps(e, r, pm, m, 1);
        const DModel& h = pm.host[0];
        Staged<double> dc, de;
        dc.make((size_t)nconfs * h.conf_size, e->stream, confs);
        de.make(nconfs, e->stream);
        if (e->precision != SG_PREC_FP64) {  // the batched search's mixed-precision BFGS
            require(h.npchunks >= 0, "mixed-precision path: at most 255 atoms per model");
            const size_t ws = (ws32_bytes(h) + 15) & ~(size_t)15;
            const size_t stage =
                (size_t)stage32_bytes(h.natoms, h.nframes, h.nheavy, h.npchunks, h.nlig, h.nblocks, h.ntors);
            require(stage + (size_t)std::max(1, e->tpc / 32) * ws <= (size_t)e->max_smem,
                    "model too large for the mixed-precision path's shared memory");
            cuda_check(launch_bfgs32(pm.dmodels.as<DModel>(), stage, ws, tables32(e), maps32(e, r), nconfs, dc.p(), v,
                                     slope, maxiters, accurate_line, early_term, de.p(), std::max(1, e->tpc / 32),
                                     e->stream),
                       "bfgs launch");
            dc.fetch(confs, e->stream);
            de.fetch(out_e, e->stream);
            e->check_device_errors();
            return;
        }
        require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
        cuda_check(launch_bfgs64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(), nconfs, dc.p(), v,
                                 slope, maxiters, accurate_line, early_term, de.p(), e->d_err.as<int>(), e->stream),
                   "bfgs launch");
        dc.fetch(confs, e->stream);
        de.fetch(out_e, e->stream);
        e->check_device_errors();
    });
}

int sg_dock(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const sg_chain_input* chains, int nchains,
            const sg_mc_params* p, sg_chain_result* out) {
    return guarded(e, [&] {
        require(chains && p && out && nchains > 0 && nchains <= (1 << 22), "dock: bad arguments");
        require(p->num_saved_mins >= 1 && p->num_saved_mins <= 1024 && p->maxiters >= 0 && p->temperature > 0,
                "dock: bad search parameters");
        RecState& r = receptor_for(e, rid);
        PackedModels pm;
        pack_models(e, models, nmodels, pm);
        ensure_model_maps(e, r, pm, models, nmodels);
        require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
        const int S = p->num_saved_mins;
        // per-chain inputs and result storage (one device allocation each)
        std::vector<double> conf0;
        std::vector<uint32_t> mt((size_t)nchains * 625);
        std::vector<size_t> conf_off(nchains), cres_off(nchains), xres_off(nchains);
        size_t nconf_res = 0, nxyz_res = 0;
        for (int k = 0; k < nchains; k++) {
            const sg_chain_input& c = chains[k];
            require(c.model >= 0 && c.model < nmodels && c.conf && c.mt && c.maxiters >= 0, "dock: bad chain input");
            require(c.mt[624] <= 624, "dock: mt19937 index out of range");
            const DModel& h = pm.host[c.model];
            conf_off[k] = conf0.size();
            conf0.insert(conf0.end(), c.conf, c.conf + h.conf_size);
            std::memcpy(&mt[(size_t)k * 625], c.mt, 625 * sizeof(uint32_t));
            cres_off[k] = nconf_res;
            nconf_res += (size_t)S * h.conf_size;
            xres_off[k] = nxyz_res;
            nxyz_res += (size_t)S * h.nheavy * 3;
            require(out[k].e && out[k].conf && out[k].coords, "dock: null result arrays");
        }
        Staged<double> d_conf0, d_e, d_conf, d_xyz, d_hist;
        Staged<uint32_t> d_mt;
        Staged<unsigned long long> d_histw;
        Staged<int> d_order, d_count;
        Staged<unsigned long long> d_evals;
        // QuickVina 2 histories (MCParams::visited), one block per chain whose dof fits
        std::vector<size_t> hist_off(nchains, SIZE_MAX), histw_off(nchains, SIZE_MAX);
        size_t nhist = 0, nhistw = 0;
        if (p->visited)
            for (int k = 0; k < nchains; k++) {
                const int n = pm.host[chains[k].model].dof;
                if (n > kHistMaxN) continue;
                hist_off[k] = nhist;
                histw_off[k] = nhistw;
                nhist += hist64_doubles(n);
                nhistw += hist64_words(n);
            }
        if (nhist) {
            d_hist.make(nhist, e->stream);
            d_histw.make(nhistw, e->stream);
            d_histw.zero(e->stream);  // empty histories
        }
        d_conf0.make(conf0.size(), e->stream, conf0.data());
        d_mt.make(mt.size(), e->stream, mt.data());
        d_e.make((size_t)nchains * S, e->stream);
        d_conf.make(nconf_res, e->stream);
        d_xyz.make(nxyz_res, e->stream);
        d_order.make((size_t)nchains * S, e->stream);
        d_count.make(nchains, e->stream);
        d_evals.make(nchains, e->stream);
        std::vector<Chain64> hc(nchains);
        for (int k = 0; k < nchains; k++) {
            hc[k].model = chains[k].model;
            hc[k].steps = chains[k].num_steps;
            hc[k].maxiters = chains[k].maxiters > 0 ? chains[k].maxiters : p->maxiters;
            hc[k].conf0 = d_conf0.p() + conf_off[k];
            hc[k].mt = d_mt.p() + (size_t)k * 625;
            hc[k].out_e = d_e.p() + (size_t)k * S;
            hc[k].out_conf = d_conf.p() + cres_off[k];
            hc[k].out_coords = d_xyz.p() + xres_off[k];
            hc[k].out_order = d_order.p() + (size_t)k * S;
            hc[k].out_count = d_count.p() + k;
            hc[k].evals = d_evals.p() + k;
            hc[k].hist = hist_off[k] == SIZE_MAX ? nullptr : d_hist.p() + hist_off[k];
            hc[k].hist_words = histw_off[k] == SIZE_MAX ? nullptr : d_histw.p() + histw_off[k];
        }
        DevBuf d_chains;
        d_chains.upload(hc.data(), hc.size() * sizeof(Chain64), e->stream);
        MCParams64 P;
        P.num_steps = p->num_steps;
        P.temperature = p->temperature;
        P.amplitude = p->mutation_amplitude;
        P.min_rmsd = p->min_rmsd;
        P.num_saved = S;
        for (int i = 0; i < 3; i++) { P.hunt[i] = p->hunt_cap[i]; P.auth[i] = p->authentic_v[i]; }
        P.maxiters = p->maxiters;
        P.accurate_line = p->accurate_line;
        P.early_term = p->early_term;
        P.slope = p->cache_slope;
        cuda_check(launch_mc64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(),
                               d_chains.as<Chain64>(), nchains, P, nhist > 0, e->d_err.as<int>(), e->stream),
                   "dock launch");
        std::vector<double> he((size_t)nchains * S), hconf(nconf_res), hxyz(nxyz_res);
        std::vector<int> horder((size_t)nchains * S), hcount(nchains);
        std::vector<unsigned long long> hev(nchains);
        d_e.fetch(he.data(), e->stream);
        d_conf.fetch(hconf.data(), e->stream);
        d_xyz.fetch(hxyz.data(), e->stream);
        d_order.fetch(horder.data(), e->stream);
        d_count.fetch(hcount.data(), e->stream);
        d_evals.fetch(hev.data(), e->stream);
        e->check_device_errors();
        for (int k = 0; k < nchains; k++) {
            const DModel& h = pm.host[chains[k].model];
            const int cnt = std::min(std::max(hcount[k], 0), S);
            out[k].count = cnt;
            out[k].evals = hev[k];
            for (int j = 0; j < cnt; j++) {
                const int slot = horder[(size_t)k * S + j];
                require(slot >= 0 && slot < S, "dock: corrupt result order");
                out[k].e[j] = he[(size_t)k * S + slot];
                std::memcpy(out[k].conf + (size_t)j * h.conf_size, &hconf[cres_off[k] + (size_t)slot * h.conf_size],
                            h.conf_size * sizeof(double));
                std::memcpy(out[k].coords + (size_t)j * h.nheavy * 3, &hxyz[xres_off[k] + (size_t)slot * h.nheavy * 3],
                            (size_t)h.nheavy * 3 * sizeof(double));
            }
        }
    });
}

int sg_refine(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const int* pose_model, int nposes,
              double* confs, const double cap[3], int maxiters, int accurate_line, int early_term, double* out_e,
              double* out_coords) {
    return guarded(e, [&] {
        require(pose_model && confs && cap && out_e && nposes > 0 && maxiters >= 0, "refine: bad arguments");
        RecState& r = receptor_for(e, rid);
        ensure_cells(e, r);
        PackedModels pm;
        pack_models(e, models, nmodels, pm);
        require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
        for (int k = 0; k < nposes; k++) require(pose_model[k] >= 0 && pose_model[k] < nmodels, "refine: bad pose model");
        const int cs = pm.max_conf, hs = pm.max_heavy;
        Staged<double> dc, de, dx;
        Staged<int> dpm;
        dc.make((size_t)nposes * cs, e->stream, confs);
        de.make(nposes, e->stream);
        dx.make((size_t)nposes * hs * 3, e->stream);
        dx.zero(e->stream);  // atoms past a pose's heavy count stay 0
        dpm.make(nposes, e->stream, pose_model);
        cuda_check(launch_refine64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(), dpm.p(), nposes,
                                   dc.p(), cs, cap, maxiters, nullptr, nullptr, accurate_line, early_term, de.p(), dx.p(), hs,
                                   e->d_err.as<int>(), e->stream),
                   "refine launch");
        dc.fetch(confs, e->stream);
        de.fetch(out_e, e->stream);
        if (out_coords) dx.fetch(out_coords, e->stream);
        e->check_device_errors();
    });
}

int sg_pair_schedule(const sg_model_desc* m, uint32_t* out, int cap, int* nchunks) {
    if (!m || !nchunks || cap < 0 || (cap > 0 && !out)) return SG_ERR_ARG;
    try {
        const int N = m->num_atoms, P = m->num_pairs;
        if (N <= 0 || P < 0 || (P > 0 && (!m->pairs || !m->atom_type))) return SG_ERR_ARG;
        std::vector<int> pair_tp(P);
        for (int k = 0; k < P; k++) {
            const int a = m->pairs[2 * k], b = m->pairs[2 * k + 1];
            if (a < 0 || a >= N || b < 0 || b >= N || a == b) return SG_ERR_ARG;
            const int ta = m->atom_type[a], tb = m->atom_type[b];
            if (ta < 0 || tb < 0 || ta >= kNumTypes || tb >= kNumTypes) return SG_ERR_ARG;
            pair_tp[k] = (ta <= tb ? tri_index(ta, tb) : tri_index(tb, ta)) | (ta > tb ? (1 << 30) : 0);
        }
        std::vector<uint32_t> slots;
        if (!pack_pair_chunks(*m, pair_tp, slots)) return SG_ERR_ARG;
        *nchunks = (int)(slots.size() / 32);
        if ((size_t)cap >= slots.size()) std::copy(slots.begin(), slots.end(), out);
        return SG_OK;
    } catch (...) {
        return SG_ERR_ARG;
    }
}

int sg_score(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const int* pose_model, int nposes,
             const double* confs, int conf_stride, const double v[3], double slope, double* out_e, double* out_intra,
             double* out_coords, int coord_stride) {
    return guarded(e, [&] {
        require(pose_model && confs && v && out_e && out_intra && nposes > 0 && nposes <= (1 << 24),
                "score: bad arguments");
        require(e->has_tables, "no tables set");
        RecState& r = receptor_for(e, rid);
        ensure_cells(e, r);
        PackedModels pm;
        pack_models(e, models, nmodels, pm);
        require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
        require(conf_stride >= pm.max_conf && (!out_coords || coord_stride >= pm.max_heavy), "score: strides too small");
        for (int k = 0; k < nposes; k++) require(pose_model[k] >= 0 && pose_model[k] < nmodels, "score: bad pose model");
        Staged<double> dc, de, di, dx;
        Staged<int> dpm;
        dc.make((size_t)nposes * conf_stride, e->stream, confs);
        de.make(nposes, e->stream);
        di.make(nposes, e->stream);
        if (out_coords) {
            dx.make((size_t)nposes * coord_stride * 3, e->stream);
            dx.zero(e->stream);  // atoms past a pose's heavy count stay 0
        }
        dpm.make(nposes, e->stream, pose_model);
        cuda_check(launch_score64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(), dpm.p(),
                                  nposes, dc.p(), conf_stride, v, slope, de.p(), di.p(), out_coords ? dx.p() : nullptr,
                                  coord_stride, e->d_err.as<int>(), e->stream),
                   "score launch");
        de.fetch(out_e, e->stream);
        di.fetch(out_intra, e->stream);
        if (out_coords) dx.fetch(out_coords, e->stream);
        e->check_device_errors();
    });
}

int sg_minimize(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const int* pose_model, int nposes,
                double* confs, int conf_stride, const double* boxes, const double cap[3], const int* maxiters,
                int accurate_line, int early_term, double* out_e, double* out_coords, int coord_stride) {
    return guarded(e, [&] {
        require(pose_model && confs && cap && maxiters && out_e && nposes > 0, "minimize: bad arguments");
        RecState& r = receptor_for(e, rid);
        ensure_cells(e, r);
        PackedModels pm;
        pack_models(e, models, nmodels, pm);
        require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
        require(conf_stride >= pm.max_conf && coord_stride >= pm.max_heavy, "minimize: strides too small");
        for (int k = 0; k < nposes; k++) {
            require(pose_model[k] >= 0 && pose_model[k] < nmodels && maxiters[k] >= 0, "minimize: bad pose");
            if (boxes)  // a pose's box must lie inside the receptor's, where its cell lists are
                for (int d = 0; d < 3; d++)
                    require(boxes[6 * k + d] >= r.gd.begin[d] && boxes[6 * k + 3 + d] <= r.gd.end[d] &&
                                boxes[6 * k + d] <= boxes[6 * k + 3 + d],
                            "minimize: a pose's box must lie inside the receptor's box");
        }
        Staged<double> dc, de, dx, db;
        Staged<int> dpm, dmi;
        dc.make((size_t)nposes * conf_stride, e->stream, confs);
        de.make(nposes, e->stream);
        dx.make((size_t)nposes * coord_stride * 3, e->stream);
        dx.zero(e->stream);  // atoms past a pose's heavy count stay 0
        dpm.make(nposes, e->stream, pose_model);
        dmi.make(nposes, e->stream, maxiters);
        if (boxes) db.make((size_t)nposes * 6, e->stream, boxes);
        cuda_check(launch_refine64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(), dpm.p(),
                                   nposes, dc.p(), conf_stride, cap, 0, dmi.p(), boxes ? db.p() : nullptr,
                                   accurate_line, early_term, de.p(), dx.p(), coord_stride, e->d_err.as<int>(),
                                   e->stream),
                   "minimize launch");
        dc.fetch(confs, e->stream);
        de.fetch(out_e, e->stream);
        if (out_coords) dx.fetch(out_coords, e->stream);
        e->check_device_errors();
    });
}

}  // extern "C"
