// Stand-in for TITAN/source/Header.h used ONLY by the oracle recipe
// (oracle/Makefile) to compile the reference's TITAN/source/Phys_param.cpp
// in place, without Boost, CGAL, Eigen or the mesh classes.
//
// The recipe passes `-I oracle/shim -I- -I <reference>/TITAN/source`, so
// `#include "Header.h"` in the reference's Phys_param.h resolves here while
// Phys_param.h itself comes from the reference tree.
//
// The physical constants and helper macros below must hold the same values as
// the reference's (TITAN/source/Header.h:20-32 and :96-104), since the Riemann
// solver reads them; they are restated, not included.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <optional>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <variant>
#include <vector>

#include "Eigen/Dense"

#define kv(x) ((x) * (x))
#define kvv(x, y, z) ((x) * (x) + (y) * (y) + (z) * (z))
#define norm2(x, y, z) (sqrt(kvv(x, y, z)))
#define whach(x) cout << #x << ": " << (x) << endl

const double const_pi = 3.14159265358979323846;
const double cpi4 = 4.0 * const_pi;
const double cpi8 = 8.0 * const_pi;
const double spi4 = sqrt(cpi4);
const double eps = 1E-12;
const double epsb = 1E-4;
const double eps_p = 1E-6;
const double eps_d = 1E-3;
const double MF_meDmp = (1.0 / 1836.15);

using namespace std;

// Helpers the solver calls from TITAN/source/Help_funk.cpp:219-249; the
// oracle's wrapper (oracle/ref_chlld_wrap.cpp) defines them.
void get_bazis(const Eigen::Vector3d& n, Eigen::Vector3d& t, Eigen::Vector3d& m);
double scalarProductFast(const double& ax, const double& ay, const double& az,
                         const double& bx, const double& by, const double& bz);
