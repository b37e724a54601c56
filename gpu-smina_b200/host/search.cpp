/*
 * Search parameters and chain seeding.
 *   setup_search            main.cpp:513-529
 *   parallel_mc seeding     parallel_mc.cpp:80-98 (random_int(0, 1000000) per task)
 *   conf::randomize         conf.h:355-360, rigid_conf::randomize conf.h:104-107
 *   mt19937 / uniform_real / uniform_int with Boost semantics (random.cpp:28-60)
 * The start orientation draws its four normals with the Marsaglia polar
 * method (Marsaglia & Bray 1964) instead of Boost's normal_distribution;
 * every consumer (device chains and the CPU checker) starts from the same
 * host-made conf and generator state, so runs stay comparable bit for bit.
 */
#include "sg_host.h"
#include <cmath>
#include <cstring>
#include <limits>

namespace sgh {

unsigned search_steps(const Model& m) {
    size_t heuristic = (size_t)m.num_movable + 10 * (size_t)m.dof;
    return unsigned(70 * 3 * (50 + heuristic) / 2);
}

// --fast's chain split (not smina's search), gpu_docking.cpp:87-112,168-220:
// every task becomes `split` chains with ceil(steps * fraction / split) steps.
// Automatic split (chain_split 0): the largest power of two from 32 down to
// 4 whose chains stay within 4 waves of the device's resident capacity.
// Automatic fraction (step_fraction 0): 1/2 for splits from 4 up to 31
// (the device is full), else 1.  A first-pass budget > 0 overrides the
// fraction.
FastPlan fast_plan(size_t tasks, size_t capacity, int chain_split, double step_fraction, double budget,
                   unsigned steps) {
    FastPlan f;
    if (chain_split > 0) {
        f.split = chain_split;
    } else {
        f.split = 32;
        while (f.split > 4 && tasks * (size_t)f.split > 4 * capacity) f.split /= 2;
    }
    f.fraction = budget > 0 ? budget : step_fraction > 0 ? step_fraction : (f.split >= 4 && f.split < 32 ? 0.5 : 1.0);
    const double per = std::ceil(steps * f.fraction / f.split);
    f.steps = per < 1 ? 1u : unsigned(per);
    return f;
}

sg_mc_params search_params(const Model& m, int num_modes) {
    sg_mc_params p{};  // visited = 0: smina's search
    p.num_steps = search_steps(m);
    p.temperature = 1.2;
    p.mutation_amplitude = 2;
    p.min_rmsd = 1.0;
    p.num_saved_mins = num_modes > 20 ? num_modes : 20;
    for (int i = 0; i < 3; i++) { p.hunt_cap[i] = 10; p.authentic_v[i] = 1000; }
    p.maxiters = (int)((25 + (size_t)m.num_movable) / 3);
    p.accurate_line = 0;
    p.early_term = 0;
    p.cache_slope = 1e6;
    return p;
}

void MT::seed(uint32_t s) {
    x[0] = s;
    for (int k = 1; k < 624; k++) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
    i = 624;
}
uint32_t MT::next() {
    if (i >= 624) {
        const uint32_t hi = 0x80000000u, lo = 0x7fffffffu, a = 0x9908b0dfu;
        for (int k = 0; k < 624; k++) {
            uint32_t y = (x[k] & hi) | (x[(k + 1) % 624] & lo);
            x[k] = x[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        i = 0;
    }
    uint32_t z = x[i++];
    z ^= z >> 11;
    z ^= (z << 7) & 0x9d2c5680u;
    z ^= (z << 15) & 0xefc60000u;
    z ^= z >> 18;
    return z;
}
double random_fl(double a, double b, MT& g) {
    for (;;) {
        double r = (double)g.next() / (4294967295.0 + 1) * (b - a) + a;
        if (r < b) return r;
    }
}
int random_int(int a, int b, MT& g) {
    uint32_t range = (uint32_t)b - (uint32_t)a;
    if (range == 0) return a;
    const uint32_t brange = 0xffffffffu;
    uint32_t bucket = brange / (range + 1);
    if (brange % (range + 1) == range) ++bucket;
    for (;;) {
        uint32_t r = g.next() / bucket;
        if (r <= range) return (int)(r + (uint32_t)a);
    }
}
double random_normal(MT& g) {
    for (;;) {
        double u = random_fl(-1, 1, g), v = random_fl(-1, 1, g);
        double s = u * u + v * v;
        if (s >= 1 || s == 0) continue;
        return u * std::sqrt(-2.0 * std::log(s) / s);
    }
}

ChainStart make_chain(const Model& m, uint32_t seed, const sg_grid_dims& box) {
    ChainStart c;
    c.conf.assign(m.conf_size, 0.0);
    MT g;
    g.seed(seed);
    const double eps = std::numeric_limits<double>::epsilon();
    for (size_t f = 0; f < m.fkind.size(); f++) {
        if (m.fkind[f] == SG_FRAME_RIGID) {
            double* x = &c.conf[m.fconf[f]];
            for (int i = 0; i < 3; i++) x[i] = random_fl(box.begin[i], box.end[i], g);
            for (;;) {
                double q[4];
                for (int k = 0; k < 4; k++) q[k] = random_normal(g);
                double nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
                if (nrm > eps) {
                    for (int k = 0; k < 4; k++) x[3 + k] = q[k] / nrm;
                    break;
                }
            }
            // this ligand's torsions, in order (ligand_conf::randomize)
            int tors = 0;
            for (size_t h = f + 1; h < m.fkind.size() && m.fkind[h] == SG_FRAME_SEGMENT; h++) tors++;
            for (int k = 0; k < tors; k++) x[7 + k] = random_fl(-3.1415926535897931, 3.1415926535897931, g);
        }
    }
    for (size_t f = 0; f < m.fkind.size(); f++)  // residue_conf::randomize
        if (m.fkind[f] != SG_FRAME_RIGID) {
            bool flex = false;
            for (int p = (int)f; p >= 0; p = m.fparent[p]) flex |= m.fkind[p] == SG_FRAME_FIRST_SEGMENT;
            if (flex) c.conf[m.fconf[f]] = random_fl(-3.1415926535897931, 3.1415926535897931, g);
        }
    std::memcpy(c.mt, g.x, sizeof(g.x));
    c.mt[624] = (uint32_t)g.i;
    return c;
}

std::vector<ChainStart> seed_chains(const Model& m, int seed, int tasks, const sg_grid_dims& box) {
    MT gen;
    gen.seed((uint32_t)seed);
    std::vector<ChainStart> out;
    for (int i = 0; i < tasks; i++) out.push_back(make_chain(m, (uint32_t)random_int(0, 1000000, gen), box));
    return out;
}

}  // namespace sgh
