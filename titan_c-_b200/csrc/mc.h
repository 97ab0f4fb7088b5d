// Monte-Carlo neutral tracing (mc_neutral.cu): arguments, the per-cell record
// the tracer reads, and the launchers.
#pragma once
#include <cuda_runtime.h>

#include "step_types.h"

namespace titan {

// Tabulated inflow distributions (titan_set_mc_face_dist) in device numbering:
// index[f] = the table of face f or -1; per table the AMR_f frame, the side
// the neutrals enter, the inflow per unit area (sum of box volume * f * |x_c|
// over the leaves) and its leaves; per leaf its box and the face's
// cumulative share of the inflow up to it (the last leaf of a face holds 1).
struct McFaceDist {
    const int* index;        // [nface], or null: no tables
    const double* frame;     // [ntab][9] Vn, Vt, Vm
    const signed char* side; // [ntab]
    const double* flux;      // [ntab] inflow per unit face area
    const int* leaf_ptr;     // [ntab + 1]
    const double* box;       // [nleaf][6]
    const double* cum;       // [nleaf]
};

// Tallied outgoing distributions (titan_set_mc_face_tally) in device
// numbering: a neutral that reaches a listed face from the table's side cell
// stops there and adds its weight to the leaf holding its local velocity
// (clamped into the table's bounds), and mu / |v_n|, mu, mu / v_n^2 to the
// face's moments. The pack kernel marks such a face in the side cell's record
// as neighbour -3 - table.
struct McFaceTally {
    const int* index;        // [nface], or null: no tallies
    const int* face;         // [ntab] device face ids
    const signed char* side; // [ntab]
    const double* frame;     // [ntab][9] Vn, Vt, Vm
    const double* bounds;    // [ntab][6] the leaves' bounding box
    const int* leaf_ptr;     // [ntab + 1]
    const double* box;       // [nleaf][6]
    double* f;               // [nleaf] summed weights
    double* mom;             // [ntab][3] n, Smu, nn
    unsigned long long* unplaced;  // neutrals whose velocity no leaf holds
};

struct McArgs {
    MeshView M;
    Params P;
    Layer L;                  // current geometry (face centres / normals, cell volumes)
    const double* state;      // [ns][ncell]
    const double* inflow_cdf; // [nface] share of the inflow through faces 0..f, last = 1
    long long nparticles;
    double mu;                // weight: inflow rate per particle
    double nH, uH0, uH1, uH2, cpH;
    unsigned face_types;      // bit t set: faces of type t let neutrals in
    unsigned long long seed;
    int max_cells;
    double* tally;            // [5][ncell]: sum mu*t, sum mu*dv (3), sum mu*d(v^2)/2
    unsigned long long* lost;
    double* trace;            // null, or [nparticles][8]: each neutral's end (titan_mc_params.trace_out)
    McFaceDist fd;            // tabulated inflow of some faces (fd.index null: none)
    McFaceTally ft;           // tallied outflow of some faces (ft.index null: none)
};

// One cell's tracing record, built once per Monte-Carlo pass: the six face
// planes (outward normal, normal . face centre), the neighbour across each
// face (-1 on the boundary), and the proton fluid the neutrals exchange with.
// One 256-byte record per crossing replaces three dependent lookups (cell ->
// faces -> face geometry and neighbour).
struct alignas(16) McCell {
    double plane[6][4];  // n0, n1, n2, d
    int nbr[6];
    double rho_th, cp;
    double V[3];
};
static_assert(sizeof(McCell) == 256, "McCell is one 256-byte record");

// Faces per block of the inflow scan, and the block-sum buffer it needs.
constexpr int kMcScanChunk = 4096;
inline int mc_scan_blocks(long long nface) { return (int)((nface + kMcScanChunk - 1) / kMcScanChunk); }

// cdf[f] = (inflow through faces 0..f) / total, total = *total_out: the flux of
// the drifting Maxwellian (nH, uH, cpH) through the inward normal of every face
// whose type is in a.face_types, times its area. The sums run in a fixed order,
// so a pass is reproducible. block_sums holds mc_scan_blocks(nface) doubles.
cudaError_t launch_mc_inflow_cdf(const McArgs& a, double* cdf, double* block_sums, double* total_out,
                                 cudaStream_t s);
cudaError_t launch_mc_pack(const McArgs& a, McCell* cells, cudaStream_t s);
cudaError_t launch_mc_trace_cells(const McArgs& a, const McCell* cells, cudaStream_t s);
cudaError_t launch_mc_normalise(double* tally, const double* vol, int ncell, cudaStream_t s);
// The outgoing tables' weights and moments per unit face area, and the
// weights per unit box volume and normal speed (AMR_f::Normir_velocity_volume).
cudaError_t launch_mc_tally_normalise(const McArgs& a, int ntab, cudaStream_t s);

}  // namespace titan
