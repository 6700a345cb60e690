// GENERATED by spin_colour_kernel_b200/gen_lattices.py from crystals.make: do not edit by hand.
// Compile-time bond tables (one coupling group per shell) of the specialised class kernels.
#pragma once

#include <stdint.h>

namespace sck {

struct BondC {
  int a2, dx, dy, dz;
};

// square, shells (1,): b = 1, D = 2, reach 1
struct Lat_square_1 {
  static constexpr int id = 1;
  static constexpr int b = 1;
  static constexpr int dim = 2;
  static constexpr int reach = 1;
  static constexpr int groups = 1;
  static constexpr int max_bonds = 4;
  __host__ __device__ static constexpr int n_bonds(int a) {
    constexpr int t[1] = {4};
    return t[a];
  }
  __host__ __device__ static constexpr int group_end(int a, int g) {
    constexpr int t[1][1] = {{4}};
    return t[a][g];
  }
  __host__ __device__ static constexpr BondC bond(int a, int i) {
    constexpr BondC t[1][4] = {
        {{0, -1, 0, 0}, {0, 0, -1, 0}, {0, 0, 1, 0}, {0, 1, 0, 0}},
    };
    return t[a][i];
  }
};

// triangular, shells (1,): b = 1, D = 2, reach 1
struct Lat_triangular_1 {
  static constexpr int id = 2;
  static constexpr int b = 1;
  static constexpr int dim = 2;
  static constexpr int reach = 1;
  static constexpr int groups = 1;
  static constexpr int max_bonds = 6;
  __host__ __device__ static constexpr int n_bonds(int a) {
    constexpr int t[1] = {6};
    return t[a];
  }
  __host__ __device__ static constexpr int group_end(int a, int g) {
    constexpr int t[1][1] = {{6}};
    return t[a][g];
  }
  __host__ __device__ static constexpr BondC bond(int a, int i) {
    constexpr BondC t[1][6] = {
        {{0, -1, 0, 0}, {0, -1, 1, 0}, {0, 0, -1, 0}, {0, 0, 1, 0}, {0, 1, -1, 0}, {0, 1, 0, 0}},
    };
    return t[a][i];
  }
};

// sc, shells (1,): b = 1, D = 3, reach 1
struct Lat_sc_1 {
  static constexpr int id = 3;
  static constexpr int b = 1;
  static constexpr int dim = 3;
  static constexpr int reach = 1;
  static constexpr int groups = 1;
  static constexpr int max_bonds = 6;
  __host__ __device__ static constexpr int n_bonds(int a) {
    constexpr int t[1] = {6};
    return t[a];
  }
  __host__ __device__ static constexpr int group_end(int a, int g) {
    constexpr int t[1][1] = {{6}};
    return t[a][g];
  }
  __host__ __device__ static constexpr BondC bond(int a, int i) {
    constexpr BondC t[1][6] = {
        {{0, -1, 0, 0}, {0, 0, -1, 0}, {0, 0, 0, -1}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 1, 0, 0}},
    };
    return t[a][i];
  }
};

// bcc, shells (1,): b = 2, D = 3, reach 1
struct Lat_bcc_1 {
  static constexpr int id = 4;
  static constexpr int b = 2;
  static constexpr int dim = 3;
  static constexpr int reach = 1;
  static constexpr int groups = 1;
  static constexpr int max_bonds = 8;
  __host__ __device__ static constexpr int n_bonds(int a) {
    constexpr int t[2] = {8, 8};
    return t[a];
  }
  __host__ __device__ static constexpr int group_end(int a, int g) {
    constexpr int t[2][1] = {{8}, {8}};
    return t[a][g];
  }
  __host__ __device__ static constexpr BondC bond(int a, int i) {
    constexpr BondC t[2][8] = {
        {{1, -1, -1, -1}, {1, -1, -1, 0}, {1, -1, 0, -1}, {1, -1, 0, 0}, {1, 0, -1, -1}, {1, 0, -1, 0}, {1, 0, 0, -1}, {1, 0, 0, 0}},
        {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 0, 1, 1}, {0, 1, 0, 0}, {0, 1, 0, 1}, {0, 1, 1, 0}, {0, 1, 1, 1}},
    };
    return t[a][i];
  }
};

// bcc, shells (1, 2): b = 2, D = 3, reach 1
struct Lat_bcc_1_2 {
  static constexpr int id = 5;
  static constexpr int b = 2;
  static constexpr int dim = 3;
  static constexpr int reach = 1;
  static constexpr int groups = 2;
  static constexpr int max_bonds = 14;
  __host__ __device__ static constexpr int n_bonds(int a) {
    constexpr int t[2] = {14, 14};
    return t[a];
  }
  __host__ __device__ static constexpr int group_end(int a, int g) {
    constexpr int t[2][2] = {{8, 14}, {8, 14}};
    return t[a][g];
  }
  __host__ __device__ static constexpr BondC bond(int a, int i) {
    constexpr BondC t[2][14] = {
        {{1, -1, -1, -1}, {1, -1, -1, 0}, {1, -1, 0, -1}, {1, -1, 0, 0}, {1, 0, -1, -1}, {1, 0, -1, 0}, {1, 0, 0, -1}, {1, 0, 0, 0}, {0, -1, 0, 0}, {0, 0, -1, 0}, {0, 0, 0, -1}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 1, 0, 0}},
        {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 0, 1, 1}, {0, 1, 0, 0}, {0, 1, 0, 1}, {0, 1, 1, 0}, {0, 1, 1, 1}, {1, -1, 0, 0}, {1, 0, -1, 0}, {1, 0, 0, -1}, {1, 0, 0, 1}, {1, 0, 1, 0}, {1, 1, 0, 0}},
    };
    return t[a][i];
  }
};

// fcc, shells (1,): b = 4, D = 3, reach 1
struct Lat_fcc_1 {
  static constexpr int id = 6;
  static constexpr int b = 4;
  static constexpr int dim = 3;
  static constexpr int reach = 1;
  static constexpr int groups = 1;
  static constexpr int max_bonds = 12;
  __host__ __device__ static constexpr int n_bonds(int a) {
    constexpr int t[4] = {12, 12, 12, 12};
    return t[a];
  }
  __host__ __device__ static constexpr int group_end(int a, int g) {
    constexpr int t[4][1] = {{12}, {12}, {12}, {12}};
    return t[a][g];
  }
  __host__ __device__ static constexpr BondC bond(int a, int i) {
    constexpr BondC t[4][12] = {
        {{1, -1, -1, 0}, {1, -1, 0, 0}, {1, 0, -1, 0}, {1, 0, 0, 0}, {2, -1, 0, -1}, {2, -1, 0, 0}, {2, 0, 0, -1}, {2, 0, 0, 0}, {3, 0, -1, -1}, {3, 0, -1, 0}, {3, 0, 0, -1}, {3, 0, 0, 0}},
        {{0, 0, 0, 0}, {0, 0, 1, 0}, {0, 1, 0, 0}, {0, 1, 1, 0}, {2, 0, 0, -1}, {2, 0, 0, 0}, {2, 0, 1, -1}, {2, 0, 1, 0}, {3, 0, 0, -1}, {3, 0, 0, 0}, {3, 1, 0, -1}, {3, 1, 0, 0}},
        {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 1, 0, 0}, {0, 1, 0, 1}, {1, 0, -1, 0}, {1, 0, -1, 1}, {1, 0, 0, 0}, {1, 0, 0, 1}, {3, 0, -1, 0}, {3, 0, 0, 0}, {3, 1, -1, 0}, {3, 1, 0, 0}},
        {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 0, 1, 1}, {1, -1, 0, 0}, {1, -1, 0, 1}, {1, 0, 0, 0}, {1, 0, 0, 1}, {2, -1, 0, 0}, {2, -1, 1, 0}, {2, 0, 0, 0}, {2, 0, 1, 0}},
    };
    return t[a][i];
  }
};

constexpr int kLatticeSpecs = 6;

}  // namespace sck
