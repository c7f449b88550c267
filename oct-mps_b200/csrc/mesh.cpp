// Mesh preprocessing: .mesh file -> face planes, orientation signs and
// adjacency in SerializeGraph's layout, plus root finding.
//
// Result-identical to MeshGraph + SerializeGraph (src/mesh.cpp:86-359) but
// O(T) instead of O(T^2): faces are matched through a hash table keyed on
// the (deduplicated) vertex coordinates instead of the reference's linear
// scan over all earlier faces (CheckFaceExists, src/mesh.cpp:51-80).  The
// arithmetic that produces planes and signs is the reference's, operation
// for operation: vertices read as float, the normal as a long-double cross
// product (V0-V1)x(V0-V2) normalised by a long-double square root rounded to
// double, d = -N.V0 in double, and the side tests against the "midpoint"
// ((((v0+v1)/2+v2)/2+v3)/2) in double.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "octmps_host.h"

namespace {

struct Vtx {
    double x, y, z;
};

struct CoordKey {
    uint64_t a, b, c;
    bool operator==(const CoordKey &o) const { return a == o.a && b == o.b && c == o.c; }
};
struct CoordHash {
    size_t operator()(const CoordKey &k) const {
        uint64_t h = k.a * 0x9e3779b97f4a7c15ull;
        h ^= k.b + 0x7f4a7c159e3779b9ull + (h << 6) + (h >> 2);
        h ^= k.c + 0x94d049bb133111ebull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

inline uint64_t dbits(double v) {
    v += 0.0;  // -0.0 and +0.0 compare equal in the reference
    uint64_t u;
    memcpy(&u, &v, 8);
    return u;
}

// Open-addressing table: sorted canonical vertex triple -> face index.
struct FaceTable {
    struct Slot {
        uint32_t v0, v1, v2;
        int32_t face;  // -1 = empty
    };
    std::vector<Slot> slots;
    uint64_t mask;
    explicit FaceTable(uint64_t expected) {
        uint64_t cap = 16;
        while (cap < 2 * expected) cap <<= 1;
        slots.assign(cap, Slot{0, 0, 0, -1});
        mask = cap - 1;
    }
    static uint64_t hash(uint32_t a, uint32_t b, uint32_t c) {
        uint64_t h = ((uint64_t)a * 0x9e3779b97f4a7c15ull) ^ ((uint64_t)b * 0xc2b2ae3d27d4eb4full) ^
                     ((uint64_t)c * 0x165667b19e3779f9ull);
        h ^= h >> 29;
        h *= 0xbf58476d1ce4e5b9ull;
        h ^= h >> 32;
        return h;
    }
    int32_t find(uint32_t a, uint32_t b, uint32_t c) const {
        for (uint64_t i = hash(a, b, c) & mask;; i = (i + 1) & mask) {
            const Slot &s = slots[i];
            if (s.face < 0) return -1;
            if (s.v0 == a && s.v1 == b && s.v2 == c) return s.face;
        }
    }
    void insert(uint32_t a, uint32_t b, uint32_t c, int32_t face) {
        for (uint64_t i = hash(a, b, c) & mask;; i = (i + 1) & mask) {
            Slot &s = slots[i];
            if (s.face < 0) {
                s = Slot{a, b, c, face};
                return;
            }
            if (s.v0 == a && s.v1 == b && s.v2 == c) return;  // keep the first
        }
    }
};

inline void sort3(uint32_t &a, uint32_t &b, uint32_t &c) {
    if (a > b) std::swap(a, b);
    if (b > c) std::swap(b, c);
    if (a > b) std::swap(a, b);
}

// readints / readfloats of src/octmps_io.cpp:444-494.
struct Reader {
    FILE *f;
    template <typename V>
    bool read(const char *fmt, int want, V *out, int bufsize) {
        char line[257];
        int ii = 0;
        while (ii <= 0) {
            if (feof(f)) return false;
            if (!fgets(line, bufsize, f)) return false;
            V tmp[5] = {0, 0, 0, 0, 0};
            ii = sscanf(line, fmt, &tmp[0], &tmp[1], &tmp[2], &tmp[3], &tmp[4]);
            if (ii > want) return false;
            if (ii > 0)
                for (int k = 0; k < 5; ++k) out[k] = tmp[k];
        }
        return true;
    }
};

}  // namespace

extern "C" void octmps_mesh_host_free(octmps_host_mesh *m) {
    if (!m) return;
    free(m->tet_region);
    free(m->tet_faces);
    free(m->tet_signs);
    free(m->tet_adj);
    free(m->face_plane);
    memset(m, 0, sizeof *m);
}

extern "C" octmps_status octmps_mesh_build_file(const char *path, octmps_host_mesh *out) {
    if (!path || !out) return OCTMPS_ERR_INVALID_ARG;
    memset(out, 0, sizeof *out);
    FILE *f = fopen(path, "r");
    if (!f) return OCTMPS_ERR_IO;
    Reader r{f};
    int it[5];
    float ft[5];
    if (!r.read("%d %d %d %d %d", 1, it, 256)) { fclose(f); return OCTMPS_ERR_IO; }
    const int nv = it[0];
    if (!r.read("%d %d %d %d %d", 1, it, 256)) { fclose(f); return OCTMPS_ERR_IO; }
    const int nt = it[0];
    if (nv < 4 || nt < 1 || nt > (1 << 28)) { fclose(f); return OCTMPS_ERR_INVALID_ARG; }

    std::vector<Vtx> verts(nv);
    std::vector<uint32_t> canon(nv);  // first vertex index with the same coordinates
    {
        std::unordered_map<CoordKey, uint32_t, CoordHash> seen;
        seen.reserve((size_t)nv * 2);
        for (int i = 0; i < nv; ++i) {
            if (!r.read("%f %f %f %f %f", 3, ft, 200)) { fclose(f); return OCTMPS_ERR_IO; }
            verts[i] = Vtx{ft[0], ft[1], ft[2]};
            CoordKey k{dbits(verts[i].x), dbits(verts[i].y), dbits(verts[i].z)};
            auto ins = seen.emplace(k, (uint32_t)i);
            canon[i] = ins.first->second;
        }
    }
    std::vector<int32_t> tv(4 * (size_t)nt), region(nt);
    for (int i = 0; i < nt; ++i) {
        if (!r.read("%d %d %d %d %d", 5, it, 256)) { fclose(f); return OCTMPS_ERR_IO; }
        for (int k = 0; k < 4; ++k) {
            if (it[k] < 1 || it[k] > nv) { fclose(f); return OCTMPS_ERR_INVALID_ARG; }
            tv[4 * (size_t)i + k] = it[k] - 1;
        }
        region[i] = it[4];
    }
    fclose(f);

    static const int combo[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const size_t nf_slots = 4 * (size_t)nt;
    std::vector<double> G;  // unoriented planes as first computed, 4 per face
    G.reserve(nf_slots * 2);
    std::vector<int32_t> intro_tet;
    std::vector<int32_t> tface(4 * (size_t)nt), adj(4 * (size_t)nt, -1);
    FaceTable table(2 * (size_t)nt + 16);
    int32_t n_distinct = 0;
    for (int i = 0; i < nt; ++i) {
        const int32_t *v = &tv[4 * (size_t)i];
        int32_t found[4] = {-1, -1, -1, -1};
        uint32_t key[4][3];
        for (int j = 0; j < 4; ++j) {
            uint32_t a = canon[v[combo[j][0]]], b = canon[v[combo[j][1]]], c = canon[v[combo[j][2]]];
            sort3(a, b, c);
            key[j][0] = a;
            key[j][1] = b;
            key[j][2] = c;
            if (i > 0) found[j] = table.find(a, b, c);
        }
        for (int j = 0; j < 4; ++j) {
            if (found[j] == -1) {
                const Vtx &V0 = verts[v[combo[j][0]]];
                const Vtx &V1 = verts[v[combo[j][1]]];
                const Vtx &V2 = verts[v[combo[j][2]]];
                // Crossproduct, src/mesh.cpp:6-12, arguments (V0-V1), (V0-V2).
                const long double x1 = V0.x - V1.x, y1 = V0.y - V1.y, z1 = V0.z - V1.z;
                const long double x2 = V0.x - V2.x, y2 = V0.y - V2.y, z2 = V0.z - V2.z;
                long double Nx = y1 * z2 - z1 * y2;
                long double Ny = z1 * x2 - x1 * z2;
                long double Nz = x1 * y2 - y1 * x2;
                const double norm = (double)sqrtl(Nx * Nx + Ny * Ny + Nz * Nz);
                Nx /= norm;
                Ny /= norm;
                Nz /= norm;
                const double nx = (double)Nx, ny = (double)Ny, nz = (double)Nz;
                const double mx = (double)(-Nx), my = (double)(-Ny), mz = (double)(-Nz);
                const double d = mx * V0.x + my * V0.y + mz * V0.z;
                G.push_back(nx);
                G.push_back(ny);
                G.push_back(nz);
                G.push_back(d);
                intro_tet.push_back(i);
                tface[4 * (size_t)i + j] = n_distinct;
                table.insert(key[j][0], key[j][1], key[j][2], n_distinct);
                ++n_distinct;
            } else {
                const int32_t fidx = found[j];
                const int32_t it0 = intro_tet[fidx];
                tface[4 * (size_t)i + j] = fidx;
                adj[4 * (size_t)i + j] = it0;
                // Every face of the introducing tet with the same vertex
                // coordinates gets the new neighbour (IsFacesSame loop,
                // src/mesh.cpp:207-209); more than one only in a degenerate
                // tet with coincident vertices.
                const int32_t *w = &tv[4 * (size_t)it0];
                for (int k = 0; k < 4; ++k) {
                    uint32_t a = canon[w[combo[k][0]]], b = canon[w[combo[k][1]]],
                             c = canon[w[combo[k][2]]];
                    sort3(a, b, c);
                    if (a == key[j][0] && b == key[j][1] && c == key[j][2]) adj[4 * (size_t)it0 + k] = i;
                }
            }
        }
    }

    // Orientation (src/mesh.cpp:216-245) and serialisation
    // (src/mesh.cpp:294-359): the stored plane of a face is the introducing
    // tet's copy turned to face inward; every tet gets a sign against it.
    out->n_vertices = nv;
    out->n_tets = nt;
    out->n_faces = (int32_t)nf_slots;
    out->n_distinct = n_distinct;
    out->tet_region = (int32_t *)malloc(sizeof(int32_t) * nt);
    out->tet_faces = (int32_t *)malloc(sizeof(int32_t) * 4 * nt);
    out->tet_signs = (int32_t *)malloc(sizeof(int32_t) * 4 * nt);
    out->tet_adj = (int32_t *)malloc(sizeof(int32_t) * 4 * nt);
    out->face_plane = (double *)calloc(4 * nf_slots, sizeof(double));
    if (!out->tet_region || !out->tet_faces || !out->tet_signs || !out->tet_adj || !out->face_plane) {
        octmps_mesh_host_free(out);
        return OCTMPS_ERR_OOM;
    }
    std::vector<double> mid(3 * (size_t)nt);
    for (int i = 0; i < nt; ++i) {
        const int32_t *v = &tv[4 * (size_t)i];
        double mx = 0, my = 0, mz = 0;
        mx += verts[v[0]].x;
        my += verts[v[0]].y;
        mz += verts[v[0]].z;
        for (int k = 1; k < 4; ++k) {
            mx += verts[v[k]].x;
            my += verts[v[k]].y;
            mz += verts[v[k]].z;
            mx /= 2;
            my /= 2;
            mz /= 2;
        }
        mid[3 * (size_t)i] = mx;
        mid[3 * (size_t)i + 1] = my;
        mid[3 * (size_t)i + 2] = mz;
    }
    for (int32_t fidx = 0; fidx < n_distinct; ++fidx) {
        const double *g = &G[4 * (size_t)fidx];
        const int t = intro_tet[fidx];
        const double h = g[0] * mid[3 * (size_t)t] + g[1] * mid[3 * (size_t)t + 1] +
                         g[2] * mid[3 * (size_t)t + 2] + g[3];
        const double s = h < 0 ? -1.0 : 1.0;
        double *p = &out->face_plane[4 * (size_t)fidx];
        p[0] = g[0] * s;
        p[1] = g[1] * s;
        p[2] = g[2] * s;
        p[3] = g[3] * s;
    }
    for (int i = 0; i < nt; ++i) {
        out->tet_region[i] = region[i];
        for (int k = 0; k < 4; ++k) {
            const int32_t fidx = tface[4 * (size_t)i + k];
            const double *p = &out->face_plane[4 * (size_t)fidx];
            const double h = p[0] * mid[3 * (size_t)i] + p[1] * mid[3 * (size_t)i + 1] +
                             p[2] * mid[3 * (size_t)i + 2] + p[3];
            out->tet_faces[4 * (size_t)i + k] = fidx;
            out->tet_signs[4 * (size_t)i + k] = h < 0 ? -1 : 1;
            out->tet_adj[4 * (size_t)i + k] = adj[4 * (size_t)i + k];
        }
    }
    return OCTMPS_OK;
}

// FindRootofGraph, src/mesh.cpp:257-289: the first tet (in file order)
// whose four inward planes put the probe on the inner side or on the plane,
// and whose first face through the probe is a boundary face.  A first face
// through the probe that has a neighbour is the reference's "probe is not
// placed on the surface" error.
extern "C" octmps_status octmps_mesh_find_root(const octmps_mesh_desc *m, double px, double py,
                                               double pz, int32_t *root) {
    if (!m || !root || m->n_tets < 1) return OCTMPS_ERR_INVALID_ARG;
    *root = -1;
    for (int32_t i = 0; i < m->n_tets; ++i) {
        double dist[4];
        bool inside = true;
        for (int j = 0; j < 4; ++j) {
            const int32_t f = m->tet_faces[4 * (size_t)i + j];
            const double s = (double)m->tet_signs[4 * (size_t)i + j];
            const double *p = &m->face_plane[4 * (size_t)f];
            dist[j] = px * (p[0] * s) + py * (p[1] * s) + pz * (p[2] * s) + p[3] * s;
            if (dist[j] < 0) {
                inside = false;
                break;
            }
        }
        if (!inside) continue;
        for (int j = 0; j < 4; ++j)
            if (dist[j] == 0) {
                if (m->tet_adj[4 * (size_t)i + j] == -1) {
                    *root = i;
                    return OCTMPS_OK;
                }
                return OCTMPS_ERR_NOT_FOUND;
            }
    }
    return OCTMPS_ERR_NOT_FOUND;
}
