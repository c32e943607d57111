// Synthetic SPD systems on an L x L x L node lattice with 6 unknowns per node.
//
// Every axis-neighbour edge e gets a 6x6 stiffness S_e = R R^T / 6 + 0.1 I
// with R ~ N(0,1) (scaled by 10^U(-a, a) when a > 0); [[S,-S],[-S,S]] is
// assembled into the edge's two node blocks and 1e-3 I is added on the
// diagonal. Values are accumulated in FP64 and rounded once to f32, so the
// matrix is exactly symmetric. Random numbers come from a counter-based
// splitmix64 stream keyed by (seed, edge) or (seed, row), so any node's rows
// can be generated independently and in parallel.
#include <cmath>
#include <cstring>

#include "wsb_internal.h"

namespace wsb {
namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Stream {
    uint64_t s;
    Stream(uint64_t seed, uint64_t key) : s(mix64(seed ^ mix64(key * 0xD1B54A32D192ED03ull + 1))) {}
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
};

// S = R R^T / 6 + 0.1 I (times 10^U(-a,a)) for edge key `key`.
void edge_stiffness(uint64_t seed, uint64_t key, double aniso, double S[36]) {
    Stream rng(seed, key);
    double R[36];
    for (int k = 0; k < 36; k += 2) {
        // Box-Muller on (0,1] x [0,1).
        const double u1 = 1.0 - rng.uniform(), u2 = rng.uniform();
        const double rad = std::sqrt(-2.0 * std::log(u1));
        R[k] = rad * std::cos(6.283185307179586 * u2);
        R[k + 1] = rad * std::sin(6.283185307179586 * u2);
    }
    double scale = 1.0;
    if (aniso > 0.0) scale = std::pow(10.0, (2.0 * rng.uniform() - 1.0) * aniso);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += R[i * 6 + k] * R[j * 6 + k];
            S[i * 6 + j] = (s / 6.0 + (i == j ? 0.1 : 0.0)) * scale;
        }
}

}  // namespace
}  // namespace wsb

extern "C" int wsb_lattice_sizes_get(uint32_t L, wsb_lattice_sizes *out) {
    if (!out) return WSB_ERR_BAD_INPUT;
    const uint64_t l = L;
    out->nodes = l * l * l;
    out->edges = l >= 1 ? 3 * l * l * (l - 1) : 0;
    out->n = 6 * out->nodes;
    out->bsr_blocks = out->nodes + 2 * out->edges;
    out->nnz = 36 * out->bsr_blocks;
    out->num_blocks = out->nodes;
    if (out->n > 0xffffffffull || out->nnz > 0xffffffffull) return WSB_ERR_BAD_INPUT;
    return WSB_OK;
}

extern "C" int wsb_lattice_generate(uint32_t L, uint64_t seed, double aniso, uint32_t *row_ptr, uint32_t *col,
                                    float *val, uint32_t *bs, float *b) {
    using namespace wsb;
    wsb_lattice_sizes sz;
    if (wsb_lattice_sizes_get(L, &sz) != WSB_OK || !row_ptr || !col || !val || !bs || !b) return WSB_ERR_BAD_INPUT;
    const int64_t nodes = (int64_t)sz.nodes, LL = (int64_t)L * L;
    // Node u at (x, y, z), u = x + L y + L^2 z. Neighbours in ascending index
    // order: -z, -y, -x, self, +x, +y, +z.
    auto nbrs = [&](int64_t u, int64_t *w, int *axis, int *lower) {
        const int64_t x = u % L, y = (u / L) % L, z = u / LL;
        int c = 0;
        if (z > 0) { w[c] = u - LL; axis[c] = 2; lower[c] = 1; ++c; }
        if (y > 0) { w[c] = u - L; axis[c] = 1; lower[c] = 1; ++c; }
        if (x > 0) { w[c] = u - 1; axis[c] = 0; lower[c] = 1; ++c; }
        w[c] = u; axis[c] = -1; lower[c] = 0; ++c;
        if (x + 1 < (int64_t)L) { w[c] = u + 1; axis[c] = 0; lower[c] = 0; ++c; }
        if (y + 1 < (int64_t)L) { w[c] = u + L; axis[c] = 1; lower[c] = 0; ++c; }
        if (z + 1 < (int64_t)L) { w[c] = u + LL; axis[c] = 2; lower[c] = 0; ++c; }
        return c;
    };
    // Row pointers: node u's 6 rows hold 6 * (#neighbours incl. self) entries.
    std::vector<uint64_t> node_off(nodes + 1, 0);
    for (int64_t u = 0; u < nodes; ++u) {
        int64_t w[7];
        int ax[7], lo[7];
        const int c = nbrs(u, w, ax, lo);
        node_off[u + 1] = node_off[u] + 36ull * c;
    }
    parallel_for(nodes, 2048, [&](int64_t a, int64_t e) {
        for (int64_t u = a; u < e; ++u) {
            int64_t w[7];
            int ax[7], lo[7];
            const int c = nbrs(u, w, ax, lo);
            double blocks[7][36];
            double diag[36];
            std::memset(diag, 0, sizeof diag);
            int self = 0;
            for (int k = 0; k < c; ++k) {
                if (ax[k] < 0) {
                    self = k;
                    continue;
                }
                // The edge is keyed by its lower node and axis.
                const int64_t lower_node = lo[k] ? w[k] : u;
                double S[36];
                edge_stiffness(seed, (uint64_t)lower_node * 3 + (uint64_t)ax[k] + 1, aniso, S);
                for (int q = 0; q < 36; ++q) {
                    blocks[k][q] = -S[q];
                    diag[q] += S[q];
                }
            }
            for (int i = 0; i < 6; ++i) diag[i * 6 + i] += 1e-3;
            std::memcpy(blocks[self], diag, sizeof diag);
            for (int a6 = 0; a6 < 6; ++a6) {
                const uint64_t row = 6 * (uint64_t)u + a6;
                uint64_t k0 = node_off[u] + (uint64_t)a6 * 6 * c;
                row_ptr[row] = (uint32_t)k0;
                for (int k = 0; k < c; ++k)
                    for (int j = 0; j < 6; ++j) {
                        col[k0] = (uint32_t)(6 * w[k] + j);
                        val[k0] = (float)blocks[k][a6 * 6 + j];
                        ++k0;
                    }
                Stream rb(seed, 0x4000000000000000ull + row);
                b[row] = (float)(2.0 * rb.uniform() - 1.0);
            }
            bs[u] = (uint32_t)(6 * u);
        }
    });
    row_ptr[sz.n] = (uint32_t)node_off[nodes];
    bs[nodes] = (uint32_t)sz.n;
    return WSB_OK;
}
