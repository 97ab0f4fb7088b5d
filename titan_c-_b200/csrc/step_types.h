// Plain data shared by the host side and the kernels of the plasma step.
#pragma once
#include <cstdint>

namespace titan {

constexpr int NV = 10;             // rho, Vx, Vy, Vz, p, Bx, By, Bz, Q, rho_He
constexpr double kPi = 3.14159265358979323846;
constexpr double kC8Pi = 25.13274122871834590768;  // literal of Setka_physics.cpp:1927
constexpr double kMeDmp = (1.0 / 1836.15);

// Device status word shared by all kernels of a context.
struct DevStatus {
    int err_kind;                 // 0 ok; first failure kind (see titan_b200.h)
    int err_index;                // renumbered index of the failing face/cell
    unsigned long long n_rho_floor;
    unsigned long long n_p_floor;
    unsigned long long steps_done;
    unsigned int block_counter;   // last-block-done counter of cell_update
    unsigned int pad;
    unsigned long long dt_next_bits;  // running CFL minimum (as ordered bits)
    double dt;                    // dt of the current step ("time" in Setka::Go)
    double t;                     // physical time accumulated
};

struct Params {
    double gamma, KFL, velosity_inf, omega, par_a_2, par_n_H_LISM, par_Kn, beta_switch;
    int move, soft_fixups, method_policy, npassive, nh, TS_hard, contact_hard, src_mode;
    int tvd, snos_on_hp;   // second-order faces (Phys_param::TVD, Snos_on_HP)
    int bn_in_p_on_hp;     // HP faces: magnetic pressure in p, exact gas-dynamic solver
};

struct MeshView {
    int ncell, nface, nnode, nbc;
    const int* face_c0;           // [nface] cells[0]
    const int* face_c1;           // [nface] cells[1] or -1
    const signed char* face_type; // Type_Gran
    const signed char* face_surf; // Type_Gran_surf
    const signed char* face_method;
    const int* face_bc;           // row into bc_vals or -1
    const double* bc_vals;        // [NV][nbc]
    const int* face_nodes;        // [4][nface]
    const int* cell_faces;        // [6][ncell], bit 31 set when the cell is cells[1]
    const int* cell_nodes;        // [8][ncell]
    const signed char* cell_type; // Type_cell
    const unsigned char* cell_tvd;
    const double* node_amp;       // [nnode] or null
    const double* node_phase;     // [nnode] or null
    const unsigned short* cell_fmap;  // [6][ncell]: the 4 nodes of each face slot as
                                      // 3-bit indices into the cell's 8 nodes (ALE)
    const int* face_aa;           // [nface] second-order neighbour beyond cells[0] or -1
    const int* face_bb;           // [nface] second-order neighbour beyond cells[1] or -1
    const signed char* face_nodt = nullptr;  // [nface] 1: left out of the CFL minimum, or null
};

struct Layer {  // geometry of one time layer (the reference's [2] arrays)
    double* xyz;   // [3][nnode]
    double* cc;    // [3][ncell]
    double* vol;   // [ncell]
    double* fc;    // [3][nface]
    double* fn;    // [3][nface]
    double* fa;    // [nface]
    double* fd;    // [nface] half distance between the two cell centres
};

struct FaceArgs {
    MeshView M;
    Params P;
    Layer L1;                    // geometry at the current layer
    const double* xyz2;          // node coordinates at the next layer (ALE)
    const double* state;         // [NV][ncell] current layer
    void* flux;                  // [nface][NFS] (double or float)
    DevStatus* st;
};

// What the cell update needs from the learned closure (source mode 3): this
// step's network outputs, turned into sources with the frame of the state
// they came from, and the next step's network inputs, formed from the state
// it has just written (closure.h).
struct ClosureCell {
    const float* y;              // [5][ncell] this step's network outputs (scaled units)
    uint32_t* in;                // [8][ncell] next step's input words (written)
    unsigned char* outside;      // [ncell] outside the training envelope: this step's (read), the next step's (written)
    const double* fallback;      // [4][ncell] sources of cells outside the envelope (last Monte-Carlo pass), or null
    unsigned long long* n_outside;  // cells outside the envelope this step, or null
    const float* norm;           // feature mean[8], 1/std[8], output scale[5]
    const float* env;            // [2][8] envelope (lo, hi), or null
    double nH_inf, lambda;       // cold-model proxy
    const double* cc1;           // [3][ncell] cell centres of the current layer
};

struct CellArgs {
    MeshView M;
    Params P;
    const double* vol1;
    const double* vol2;    // stationary mesh: the same volumes
    Layer L2;              // moving mesh: node coordinates of the next layer (read);
                           // its cell centres and volumes are written here
    const double* state;   // [NV][ncell] current
    double* state2;        // [NV][ncell] next
    const void* flux;
    const double* hfl;     // [5*nh][ncell] frozen neutral fluids (Bera sources)
    const double* src;     // [4][ncell] external sources (m_x, m_y, m_z, E)
    ClosureCell cl;        // source mode 3: the learned closure
    DevStatus* st;
    // [ceil(ncell / 32) + 1]: the first face whose cells[0] is >= 32 k (faces
    // sorted by cells[0], as the renumbering leaves them), so the faces owned
    // by a block of cells are one contiguous range of records; null when the
    // faces are not in that order (the staged launch shapes need it)
    const int* owner_start = nullptr;
};

}  // namespace titan
