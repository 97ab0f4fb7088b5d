// A C++ consumer of the C ABI, shaped like the binding a TITAN maintainer adds
// inside Setka: it holds the mesh as the reference's object graph (Yzel /
// Gran / Cell objects with 1-based `number`, per-object parameter maps as in
// TITAN/source/Cell.h:36 and Gran.h), flattens it the way Setka::Gpu_init
// does, steps the plasma through titan_step in place of the two OpenMP loops
// of Setka::Go (TITAN/source/Setka.h:221, Setka_physics.cpp:1634-2028) and
// copies the state back into the cell maps.
//
// Workload: the n^3 unit cube with the Brio-Wu Riemann problem along
// (1,1,0)/sqrt(2), HLLD on every face, Outer_Soft boundaries without the
// outflow fix-ups, CFL 0.4. Faces are merged the way Setka::New_connect does
// (Setka.cpp:2066-2130): each cell proposes its six quads in the reference's
// order, the first proposer becomes cells[0] and keeps its node order.
//
//   setka_consumer <n> <steps> <out.bin>
//
// out.bin (little-endian): int64 nnode, ncell, nface, steps; the flattened
// mesh (node_xyz [N][3] f64, cell_nodes [C][8] i32, cell_faces [C][6] i32,
// face_nodes [F][4] i32, face_cells [F][2] i32, face_type [F] i8); the
// initial state and the state after `steps` steps, [TITAN_NV][C] f64 each;
// f64 dt_next and t. A test replays the flattened mesh through the oracle.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "titan_b200.h"

namespace {

const char* kNames[TITAN_NV] = {"rho", "Vx", "Vy", "Vz", "p", "Bx", "By", "Bz", "Q", "rho_He"};

struct Cell;
struct Yzel {
    int number = 0;
    double coord[2][3] = {};
};
struct Gran {
    int number = 0;
    std::vector<Yzel*> yzels;
    std::vector<Cell*> cells;
    int type = 0;   // Type_Gran
    int type2 = 0;  // Type_Gran_surf
    std::map<std::string, double> parameters;
    int Get_method() const { return 3; }  // HLLD everywhere for this problem
};
struct Cell {
    int number = 0;
    std::vector<Yzel*> yzels;
    std::vector<Gran*> grans;
    int type = 0;
    bool is_TVD = true;
    std::map<std::string, double> parameters[2];
};

struct Setka {
    std::vector<Yzel*> All_Yzel;
    std::vector<Cell*> All_Cell;
    std::vector<Gran*> All_Gran;
    titan_ctx* gpu = nullptr;

    ~Setka() {
        if (gpu) titan_destroy(gpu);
        for (auto* y : All_Yzel) delete y;
        for (auto* c : All_Cell) delete c;
        for (auto* g : All_Gran) delete g;
    }

    void Build_cube(int n) {
        const int m = n + 1;
        auto nid = [m](int i, int j, int k) { return (i * m + j) * m + k; };
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                for (int k = 0; k < m; ++k) {
                    auto* y = new Yzel;
                    y->number = (int)All_Yzel.size() + 1;
                    const double x[3] = {i * (1.0 / n), j * (1.0 / n), k * (1.0 / n)};
                    for (int d = 0; d < 3; ++d) y->coord[0][d] = y->coord[1][d] = x[d];
                    All_Yzel.push_back(y);
                }
        static const int kHexFaces[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                            {2, 3, 7, 6}, {1, 2, 6, 5}, {0, 4, 7, 3}};
        std::map<std::array<int, 4>, Gran*> seen;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    auto* c = new Cell;
                    c->number = (int)All_Cell.size() + 1;
                    const int ids[8] = {nid(i, j, k),         nid(i + 1, j, k),         nid(i + 1, j + 1, k),
                                        nid(i, j + 1, k),     nid(i, j, k + 1),         nid(i + 1, j, k + 1),
                                        nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)};
                    for (int v : ids) c->yzels.push_back(All_Yzel[v]);
                    All_Cell.push_back(c);
                }
        // New_connect: faces in order of their first proposer (cell, slot)
        for (auto* c : All_Cell)
            for (auto& hf : kHexFaces) {
                std::array<int, 4> key = {c->yzels[hf[0]]->number, c->yzels[hf[1]]->number,
                                          c->yzels[hf[2]]->number, c->yzels[hf[3]]->number};
                std::array<int, 4> srt = key;
                std::sort(srt.begin(), srt.end());
                auto it = seen.find(srt);
                Gran* g;
                if (it == seen.end()) {
                    g = new Gran;
                    g->number = (int)All_Gran.size() + 1;
                    for (int v : hf) g->yzels.push_back(c->yzels[v]);
                    All_Gran.push_back(g);
                    seen[srt] = g;
                } else {
                    g = it->second;
                }
                g->cells.push_back(c);
                c->grans.push_back(g);
            }
        for (auto* g : All_Gran) g->type = g->cells.size() == 2 ? TITAN_FACE_US : TITAN_FACE_OUTER_SOFT;
    }

    // Brio-Wu along (1,1,0)/sqrt(2) in the solver's units, B stored Gaussian
    void Init_brio_wu() {
        const double spi4 = std::sqrt(4.0 * M_PI);
        const double nrm[3] = {1.0 / std::sqrt(2.0), 1.0 / std::sqrt(2.0), 0.0};
        const double tng[3] = {-1.0 / std::sqrt(2.0), 1.0 / std::sqrt(2.0), 0.0};
        for (auto* c : All_Cell) {
            double cc[3] = {0, 0, 0};
            for (auto* y : c->yzels)
                for (int d = 0; d < 3; ++d) cc[d] += y->coord[0][d];
            for (double& v : cc) v /= 8.0;
            const double s = (cc[0] - 0.5) * nrm[0] + (cc[1] - 0.5) * nrm[1] + (cc[2] - 0.5) * nrm[2];
            const bool left = s < 0.0;
            const double bt = left ? 1.0 : -1.0;
            auto& P = c->parameters[0];
            P["rho"] = left ? 1.0 : 0.125;
            P["p"] = left ? 1.0 : 0.1;
            P["Vx"] = P["Vy"] = P["Vz"] = 0.0;
            P["Bx"] = spi4 * (0.75 * nrm[0] + bt * tng[0]);
            P["By"] = spi4 * (0.75 * nrm[1] + bt * tng[1]);
            P["Bz"] = spi4 * (0.75 * nrm[2] + bt * tng[2]);
            P["Q"] = P["rho_He"] = 0.0;
            c->parameters[1] = P;
        }
    }

    // Flatten once, as the binding does after Init_physics
    bool Gpu_init(std::vector<double>& xyz, std::vector<int32_t>& cn, std::vector<int32_t>& cf,
                  std::vector<int32_t>& fn, std::vector<int32_t>& fc, std::vector<int8_t>& ft) {
        const int64_t N = All_Yzel.size(), C = All_Cell.size(), F = All_Gran.size();
        xyz.assign(3 * N, 0.0);
        cn.assign(8 * C, 0);
        cf.assign(6 * C, 0);
        fn.assign(4 * F, 0);
        fc.assign(2 * F, -1);
        ft.assign(F, 0);
        std::vector<int32_t> fb(F, -1);
        std::vector<int8_t> ct(C), fs(F);
        std::vector<uint8_t> tvd(C);
        std::vector<double> bc;
        for (auto* y : All_Yzel)
            for (int k = 0; k < 3; ++k) xyz[3 * (y->number - 1) + k] = y->coord[0][k];
        for (auto* c : All_Cell) {
            const int64_t i = c->number - 1;
            for (int k = 0; k < 8; ++k) cn[8 * i + k] = c->yzels[k]->number - 1;
            for (int k = 0; k < 6; ++k) cf[6 * i + k] = c->grans[k]->number - 1;
            ct[i] = (int8_t)c->type;
            tvd[i] = c->is_TVD;
        }
        for (auto* g : All_Gran) {
            const int64_t f = g->number - 1;
            for (int k = 0; k < 4; ++k) fn[4 * f + k] = g->yzels[k]->number - 1;
            fc[2 * f] = g->cells[0]->number - 1;
            fc[2 * f + 1] = g->cells.size() == 2 ? g->cells[1]->number - 1 : -1;
            ft[f] = (int8_t)g->type;
            fs[f] = (int8_t)g->type2;
            if (g->type == TITAN_FACE_INNER_HARD || g->type == TITAN_FACE_OUTER_HARD) {
                fb[f] = (int32_t)(bc.size() / TITAN_NV);
                for (auto* nm : kNames) bc.push_back(g->parameters[nm]);
            }
        }
        titan_mesh m{N, C, F, (int64_t)(bc.size() / TITAN_NV), xyz.data(), cn.data(), cf.data(), ct.data(),
                     tvd.data(), fn.data(), fc.data(), ft.data(), fs.data(), fb.data(),
                     bc.empty() ? nullptr : bc.data(), nullptr, nullptr};
        // Phys_param for this problem: gamma 5/3, KFL 0.4, no node motion, plain
        // Outer_Soft copies, per-face solver choice, FP64
        titan_params p{5.0 / 3.0, 0.4, -2.54327, 0.0, 0.102046, 3.0, 40.0906, 0.01,
                       /*move*/ 0, /*soft_fixups*/ 0, /*method_policy*/ 0, /*npassive*/ 0, /*nh*/ 0,
                       /*TS_hard*/ 0, /*contact_hard*/ 0, /*flux_precision*/ 64, /*tvd*/ 0, 0, 0};
        if (titan_create(&m, &p, &gpu) != TITAN_OK) {
            std::cout << titan_last_error() << std::endl;
            return false;
        }
        std::vector<int8_t> method(F);
        for (auto* g : All_Gran) method[g->number - 1] = (int8_t)g->Get_method();
        return titan_set_face_method(gpu, method.data()) == TITAN_OK;
    }

    // Setka::Go's two loops, through the library
    bool Gpu_go(size_t steps, double& time, double& t) {
        const int64_t C = All_Cell.size();
        std::vector<double> st(TITAN_NV * C);
        for (auto* c : All_Cell)
            for (int k = 0; k < TITAN_NV; ++k) st[k * C + c->number - 1] = c->parameters[0][kNames[k]];
        if (titan_upload_state(gpu, st.data()) != TITAN_OK) return false;
        titan_step_info info{};
        if (titan_step(gpu, (int64_t)steps, &time, &t, &info) != TITAN_OK) {
            std::cout << "Error " << info.err_kind << " at " << info.err_index << ": " << titan_last_error()
                      << std::endl;
            return false;
        }
        if (titan_download_state(gpu, st.data()) != TITAN_OK) return false;
        for (auto* c : All_Cell)
            for (int k = 0; k < TITAN_NV; ++k)
                c->parameters[0][kNames[k]] = c->parameters[1][kNames[k]] = st[k * C + c->number - 1];
        return true;
    }

    std::vector<double> State() {
        const int64_t C = All_Cell.size();
        std::vector<double> st(TITAN_NV * C);
        for (auto* c : All_Cell)
            for (int k = 0; k < TITAN_NV; ++k) st[k * C + c->number - 1] = c->parameters[0][kNames[k]];
        return st;
    }
};

template <typename T>
void put(FILE* f, const std::vector<T>& v) {
    fwrite(v.data(), sizeof(T), v.size(), f);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 4) {
        std::cerr << "usage: setka_consumer <n> <steps> <out.bin>" << std::endl;
        return 2;
    }
    const int n = std::atoi(argv[1]);
    const int steps = std::atoi(argv[2]);
    Setka S;
    S.Build_cube(n);
    S.Init_brio_wu();
    std::vector<double> xyz;
    std::vector<int32_t> cn, cf, fn, fc;
    std::vector<int8_t> ft;
    if (!S.Gpu_init(xyz, cn, cf, fn, fc, ft)) return 1;
    const std::vector<double> st0 = S.State();
    double time = 1e-5, t = 0.0;  // Setka::Go starts with time = 1e-5 (Setka_physics.cpp:1582)
    // two calls, as the reference's outer loop calls Go repeatedly
    if (!S.Gpu_go((size_t)(steps / 2), time, t)) return 1;
    if (!S.Gpu_go((size_t)(steps - steps / 2), time, t)) return 1;
    const std::vector<double> st1 = S.State();
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    const int64_t hdr[4] = {(int64_t)S.All_Yzel.size(), (int64_t)S.All_Cell.size(), (int64_t)S.All_Gran.size(),
                            (int64_t)steps};
    fwrite(hdr, sizeof(int64_t), 4, f);
    put(f, xyz);
    put(f, cn);
    put(f, cf);
    put(f, fn);
    put(f, fc);
    put(f, ft);
    put(f, st0);
    put(f, st1);
    fwrite(&time, sizeof(double), 1, f);
    fwrite(&t, sizeof(double), 1, f);
    std::fclose(f);
    std::cout << "setka_consumer: " << steps << " steps of the " << n << "^3 Brio-Wu cube, dt_next " << time
              << ", t " << t << std::endl;
    return 0;
}
