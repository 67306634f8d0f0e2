// The neighbourhoods as compile-time tables, shared by the sweep and the
// tally kernels.
#pragma once

namespace glz {

// The neighbour offsets of each neighbourhood in the reference's order
// (lattice.rs:8-88): a plane takes ORDER1's four in-plane faces or ORDER3's
// eight in-plane neighbours; a volume takes ORDER1, ORDER2 or ORDER3 whole.
// The host builds the same table (engine.cu) and each launch checks they agree.
template <int DIM, int NOFF>
__host__ __device__ constexpr int neighbour_offset(int k, int axis) {
    if (DIM == 2 && NOFF == 4) {
        constexpr int o[4][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
        return o[k][axis];
    }
    if (DIM == 2 && NOFF == 8) {
        constexpr int o[8][3] = {{-1, -1, 0}, {0, -1, 0}, {1, -1, 0}, {-1, 0, 0},
                                 {1, 0, 0},   {-1, 1, 0}, {0, 1, 0},  {1, 1, 0}};
        return o[k][axis];
    }
    if (DIM == 3 && NOFF == 6) {
        constexpr int o[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        return o[k][axis];
    }
    if (DIM == 3 && NOFF == 18) {
        constexpr int o[18][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                                  {1, 1, 0},  {1, -1, 0}, {-1, 1, 0},  {-1, -1, 0}, {1, 0, 1}, {1, 0, -1},
                                  {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};
        return o[k][axis];
    }
    // ORDER3: dz, then dy, then dx from -1 to 1, the centre left out
    const int kk = k < 13 ? k : k + 1;
    return axis == 0 ? kk % 3 - 1 : (axis == 1 ? (kk / 3) % 3 - 1 : kk / 9 - 1);
}

}  // namespace glz
