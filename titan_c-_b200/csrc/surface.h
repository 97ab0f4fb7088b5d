// Surface-tracking node motion (surface.cu): the device tables built by
// titan_set_surface_motion and the launcher that replaces the prescribed
// node motion of a step.
#pragma once
#include <cuda_runtime.h>

#include "step_types.h"

namespace titan {

// The A_Luch spacing law of Luch::dvigenie (TITAN/source/Luch.cpp:9-152):
// node counts and radii of Geo_param (Geo_param.h:22-63). A ray then has
// M0 + M1 + M2 + M3 + M4 + 5 nodes: M0 fixed from R0, the R1 node, M1 up to
// the TS node, M11 at the step before the TS, M2 - M11 to the HP node, M3 to
// the BS node, M4 to the outer end at R5.
struct RayLaw {
    int on;
    int M0, M1, M11, M2, M3, M4;
    double R0, R1, R5, da1, da2, da3, da4, da5;
    __host__ __device__ int ts_slot() const { return M0 + M1 + 1; }
    __host__ __device__ int hp_slot() const { return M0 + M1 + M2 + 2; }
    __host__ __device__ int bs_slot() const { return M0 + M1 + M2 + M3 + 3; }
    __host__ __device__ int length() const { return M0 + M1 + M2 + M3 + M4 + 5; }
};

struct SurfaceDev {
    // moving surface faces, grouped by surface (1 TS, 2 HP, 3 BS): positions
    // off[s] .. off[s+1]-1 of face_list hold surface s's faces (device ids)
    int off[5];
    const int* face_list;
    double* vf;             // [3][nlist]: velocity_X * ds * n of each listed face
    int nlist;
    // moving surface nodes and, per node, its faces' list positions in
    // ascending original face index
    int n_node;
    const int* node_id;     // [n_node] device node ids
    const int* node_ptr;    // [n_node + 1]
    const int* node_face;   // list positions
    // rays: device node ids from the inner end, radii and direction at the
    // start of tracking, anchors (ends and surface nodes)
    int nray, ray_len;
    const int* ray_nodes;
    const double* ray_r0;
    const double* ray_dir;  // [nray][3]
    const int2* ray_seg;    // [nray][ray_len]: slots of the anchors around a node, (-1, -1) for an anchor
    RayLaw law;             // law.on: the A_Luch law places the ray's other nodes instead
    double vel[4];          // velocity_TS / _HP / _BS at [1] / [2] / [3]
    int null_bn_on_hp;
    // smoothing of each moving node (the reference's sglag_* terms): 0 none,
    // 1 toward its fitted sphere (centre sm_centre), 2 toward the mean of it
    // and its neighbours; coefficient velocity_X * k; neighbours in ascending
    // original node order
    const signed char* sm_kind;   // [n_node]
    const double* sm_coef;        // [n_node]
    const double* sm_centre;      // [3][n_node]
    const int* nb_ptr;            // [n_node + 1]
    const int* nb_id;             // device node ids
    // [n_node] 1: an HP node that moves along (0, y, z) where x < 0 (hp_tail), or null
    const signed char* node_tail;
};

// xyz2 of `fa` from xyz of fa.L1 by surface tracking, with the step's dt from
// the status word. state_rw is fa.state, writable: null_bn_on_HP removes the
// normal B of the HP cells.
cudaError_t launch_surface_motion(const FaceArgs& fa, double* state_rw, const SurfaceDev& S, int nk, bool tvd,
                                  cudaStream_t s);

}  // namespace titan
