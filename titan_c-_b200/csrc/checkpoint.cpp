// Cell-parameter checkpoints in the reference's binary layout, so that a
// solution saved by TITAN drops into this library and back
// (Setka::Save_cell_parameters / Download_cell_parameters,
// TITAN/source/Setka_physics.cpp:4108-4231). Layout, x86-64, native endianness:
//   for each cell (the mesh's cell order):
//     size_t n; n times { size_t key_len; char key[key_len]; double value; }
//   bool has_nodes; if true: size_t nnode; nnode times { double x, y, z; }
//   1000 bytes of bool false (reserved by the writer)
// The reference writes each cell's keys in its unordered_map's order; keys are
// read in any order. Only the plasma fields this library carries are taken
// (rho, Vx, Vy, Vz, p, Bx, By, Bz, Q, rho_He); other keys (neutral fluids,
// pickup ions, Monte-Carlo tallies) are skipped, and a field missing from a
// cell leaves the caller's value in place, as Download_cell_parameters does.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/titan_b200.h"

namespace titan {
void set_last_error(const std::string& msg);
}

namespace {

const char* const kNames[TITAN_NV] = {"rho", "Vx", "Vy", "Vz", "p", "Bx", "By", "Bz", "Q", "rho_He"};

int ckfail(int code, const std::string& msg) {
    titan::set_last_error(msg);
    return code;
}

struct File {
    FILE* f = nullptr;
    explicit File(FILE* ff) : f(ff) {}
    ~File() {
        if (f) fclose(f);
    }
    template <typename T>
    bool get(T* v) {
        return fread(v, sizeof(T), 1, f) == 1;
    }
    template <typename T>
    bool put(const T& v) {
        return fwrite(&v, sizeof(T), 1, f) == 1;
    }
};

}  // namespace

extern "C" {

int titan_read_cell_parameters(const char* path, int64_t ncell, int64_t nnode, double* state, double* xyz,
                               int32_t* fields_found, int32_t* has_nodes) {
    if (!path || ncell <= 0 || !state) return ckfail(TITAN_EINVAL, "titan_read_cell_parameters: bad argument");
    File in(fopen(path, "rb"));
    if (!in.f) return ckfail(TITAN_EINVAL, std::string("titan_read_cell_parameters: cannot open ") + path);
    int32_t found = 0;
    std::vector<char> key;
    for (int64_t c = 0; c < ncell; ++c) {
        uint64_t n = 0;
        if (!in.get(&n) || n > 100000)
            return ckfail(TITAN_EINVAL, "titan_read_cell_parameters: truncated or malformed record at cell " +
                                            std::to_string(c));
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t len = 0;
            double v = 0.0;
            if (!in.get(&len) || len > 4096)
                return ckfail(TITAN_EINVAL, "titan_read_cell_parameters: malformed key at cell " + std::to_string(c));
            key.resize(len);
            if ((len && fread(key.data(), 1, len, in.f) != len) || !in.get(&v))
                return ckfail(TITAN_EINVAL, "titan_read_cell_parameters: truncated at cell " + std::to_string(c));
            for (int k = 0; k < TITAN_NV; ++k) {
                if (strlen(kNames[k]) == len && memcmp(kNames[k], key.data(), len) == 0) {
                    state[(int64_t)k * ncell + c] = v;
                    found |= 1 << k;
                    break;
                }
            }
        }
    }
    bool nodes = false;
    if (!in.get(&nodes)) nodes = false;  // files without the node block end here
    if (nodes) {
        uint64_t nn = 0;
        if (!in.get(&nn)) return ckfail(TITAN_EINVAL, "titan_read_cell_parameters: truncated node block");
        if (xyz) {
            if ((int64_t)nn != nnode)
                return ckfail(TITAN_EMESH, "titan_read_cell_parameters: file has " + std::to_string(nn) +
                                               " nodes, the mesh " + std::to_string(nnode));
            if (fread(xyz, sizeof(double), 3 * nn, in.f) != 3 * nn)
                return ckfail(TITAN_EINVAL, "titan_read_cell_parameters: truncated node block");
        }
    }
    if (fields_found) *fields_found = found;
    if (has_nodes) *has_nodes = nodes ? 1 : 0;
    return TITAN_OK;
}

int titan_write_cell_parameters(const char* path, int64_t ncell, int32_t nfields, const double* state, int64_t nnode,
                                const double* xyz) {
    if (!path || ncell <= 0 || !state || nfields < 1 || nfields > TITAN_NV || (xyz && nnode <= 0))
        return ckfail(TITAN_EINVAL, "titan_write_cell_parameters: bad argument");
    File out(fopen(path, "wb"));
    if (!out.f) return ckfail(TITAN_EINVAL, std::string("titan_write_cell_parameters: cannot open ") + path);
    bool ok = true;
    for (int64_t c = 0; c < ncell && ok; ++c) {
        ok = out.put((uint64_t)nfields);
        for (int k = 0; k < nfields && ok; ++k) {
            const uint64_t len = strlen(kNames[k]);
            ok = out.put(len) && fwrite(kNames[k], 1, len, out.f) == len && out.put(state[(int64_t)k * ncell + c]);
        }
    }
    const bool nodes = xyz != nullptr;
    ok = ok && out.put(nodes);
    if (nodes) ok = ok && out.put((uint64_t)nnode) && fwrite(xyz, sizeof(double), 3 * nnode, out.f) == (size_t)(3 * nnode);
    const bool reserved = false;
    for (int i = 0; i < 1000 && ok; ++i) ok = out.put(reserved);
    if (!ok) return ckfail(TITAN_EINVAL, std::string("titan_write_cell_parameters: write failed on ") + path);
    return TITAN_OK;
}

}  // extern "C"
