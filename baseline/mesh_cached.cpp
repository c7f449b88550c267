// The reference's mesh builder (src/mesh.cpp:86-359) replaced by a loader of
// its own output.  MeshGraph's face matching is O(T^2) in the tet count
// (about an hour at the 380,928 tets of the B-scan workload), so the
// serialised mesh and the root tet of every probe position are computed once
// on the CPU by the reference's MeshGraph + FindRootofGraph + SerializeGraph
// (oracle/ref_mesh_cache.py) and read here from the binary file named by the
// environment variable OCTMPS_REF_MESH_CACHE:
//   int32 n_tets, n_faces, n_probes
//   int32 tet[n_tets][14]   idx, region, faces[4], signs[4], adjTetras[4]
//   double face[n_faces][4] Nx, Ny, Nz, d
//   double probe_x[n_probes]
//   int32 root[n_probes]
// main() (src/main.cu:940-963) calls the three functions below with the
// signatures it expects; nothing else of the reference changes.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "octmps.h"

namespace {

struct Cache {
    int n_tets = 0, n_faces = 0, n_probes = 0;
    std::vector<int> tet;
    std::vector<double> face, xs;
    std::vector<int> roots;
    bool loaded = false;
};
Cache g_cache;
TetrahedronStruct g_stub;  // the "graph" and "root" handles main() passes around

bool load_cache() {
    if (g_cache.loaded) return true;
    const char *path = getenv("OCTMPS_REF_MESH_CACHE");
    if (!path) {
        fprintf(stderr, "OCTMPS_REF_MESH_CACHE is not set\n");
        return false;
    }
    FILE *f = fopen(path, "rb");
    if (!f) {
        perror("mesh cache");
        return false;
    }
    int hdr[3];
    bool ok = fread(hdr, sizeof(int), 3, f) == 3 && hdr[0] > 0 && hdr[1] > 0 && hdr[2] > 0;
    if (ok) {
        g_cache.n_tets = hdr[0];
        g_cache.n_faces = hdr[1];
        g_cache.n_probes = hdr[2];
        g_cache.tet.resize((size_t)hdr[0] * 14);
        g_cache.face.resize((size_t)hdr[1] * 4);
        g_cache.xs.resize(hdr[2]);
        g_cache.roots.resize(hdr[2]);
        ok = fread(g_cache.tet.data(), sizeof(int), g_cache.tet.size(), f) == g_cache.tet.size() &&
             fread(g_cache.face.data(), sizeof(double), g_cache.face.size(), f) ==
                 g_cache.face.size() &&
             fread(g_cache.xs.data(), sizeof(double), g_cache.xs.size(), f) == g_cache.xs.size() &&
             fread(g_cache.roots.data(), sizeof(int), g_cache.roots.size(), f) ==
                 g_cache.roots.size();
    }
    fclose(f);
    if (!ok) fprintf(stderr, "mesh cache %s is malformed\n", path);
    g_cache.loaded = ok;
    return ok;
}

}  // namespace

TetrahedronStruct *MeshGraph(char *filename, SimulationStruct **simulations) {
    (void)filename;
    if (!load_cache()) return NULL;
    (*simulations)->num_tetrahedrons = (short)g_cache.n_tets;  // a short, as in the reference
    return &g_stub;
}

// The cached root of the probe position main() set in (*simulations)->probe_x:
// the cached position nearest to it (positions are 10 um apart; the scan's
// double-stepped positions agree with the cache's to rounding).
TetrahedronStruct *FindRootofGraph(TetrahedronStruct *tetrahedrons, SimulationStruct **simulations) {
    (void)tetrahedrons;
    if (!load_cache()) return NULL;
    const double x = (*simulations)->probe_x;
    int best = -1;
    for (int k = 0; k < g_cache.n_probes; ++k)
        if (best < 0 || fabs(g_cache.xs[k] - x) < fabs(g_cache.xs[best] - x)) best = k;
    if (best < 0 || fabs(g_cache.xs[best] - x) > 1e-9 || g_cache.roots[best] < 0) {
        fprintf(stderr, "The probe at x=%g has no cached root\n", x);
        return NULL;
    }
    g_stub.index = g_cache.roots[best];
    return &g_stub;
}

void SerializeGraph(TetrahedronStruct *RootTetrahedron, UINT32 number_of_vertices,
                    UINT32 number_of_faces, UINT32 number_of_tetrahedrons, Vertex *d_vertices,
                    TriangleFaces *d_faces, TetrahedronStructGPU *d_root) {
    (void)RootTetrahedron;
    (void)number_of_vertices;
    (void)d_vertices;
    if (!load_cache() || (int)number_of_tetrahedrons != g_cache.n_tets ||
        (UINT32)g_cache.n_faces > number_of_faces) {
        fprintf(stderr, "mesh cache does not match the mesh file\n");
        exit(1);
    }
    for (int i = 0; i < g_cache.n_tets; ++i) {
        const int *t = &g_cache.tet[(size_t)i * 14];
        d_root[i].idx = t[0];
        d_root[i].region = t[1];
        for (int k = 0; k < 4; ++k) {
            d_root[i].faces[k] = t[2 + k];
            d_root[i].signs[k] = t[6 + k];
            d_root[i].adjTetras[k] = t[10 + k];
        }
    }
    for (UINT32 f = 0; f < number_of_faces; ++f) {
        memset(&d_faces[f], 0, sizeof(TriangleFaces));
        d_faces[f].idx = (int)f;
        if ((int)f < g_cache.n_faces) {
            d_faces[f].Nx = g_cache.face[4 * (size_t)f + 0];
            d_faces[f].Ny = g_cache.face[4 * (size_t)f + 1];
            d_faces[f].Nz = g_cache.face[4 * (size_t)f + 2];
            d_faces[f].d = g_cache.face[4 * (size_t)f + 3];
        }
    }
}
