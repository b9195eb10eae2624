// Moving air on the B200: both pressure levels carried along with the air at the start of each
// step (WaveSolver::run, cpp/include/acoustic_spaces/fdtd.hpp:833-840), by the three stages of the
// strong-stability-preserving Runge-Kutta method of fdtd.hpp:2049-2097:
//
//     t1 = q + D(q),   t2 = 3/4 q + 1/4 (t1 + D(t1)),   q <- q + 2/3 ((t2 + D(t2)) - q),
//
// D(q)_i = -v . grad q at cell i over a step, the plain way (fdtd.hpp:1946-1974: the shifts along
// x and y and four neighbour bits an axis) or round the solids (fdtd.hpp:1978-2020: each axis's
// face winds and loop terms, the border of the moving air taking only the faces that lead into it).
// Cells whose air stands still keep q at every stage. Each stage is one launch over a list of
// cells: the moving cells, then the still air cells their stencils read (the halo, whose stage
// values are q's own); both levels in one launch (blockIdx.y), each with its own stage buffers.
// Every expression keeps the reference's operands in its order, so that with T float and no
// contraction the stages round as the reference's do.
#pragma once

#include <cstdint>

namespace fdtd {

struct Flow {
    const uint32_t *cells = nullptr;  // pitched: the moving cells, then the halo
    uint32_t moving = 0, count = 0;   // moving cells; moving cells and halo
    const float *shift_x = nullptr, *shift_y = nullptr;  // plain form: cells a step along x, y
    const uint8_t *mask = nullptr;    // plain: 4 bits an axis (x low, y high); round: 0, 1, 2 (border)
    const float *wind[3] = {nullptr, nullptr, nullptr};  // round form, per axis, on each cell's + face
    const float *loop[3] = {nullptr, nullptr, nullptr};
    uint32_t sy = 0, sz = 0;          // pitched strides
    void *t1[2] = {nullptr, nullptr}, *t2[2] = {nullptr, nullptr};  // the stages, per level
};

// The plain form's gradient term along one axis of stride st (fdtd.hpp:1946-1967): the
// fourth-order central difference where both neighbours on each side are moving air (bits 0-3
// all set), else the faces that exist (an inflow or outflow face to still air by the shift's sign)
// plus the loop corrections whose cells exist.
template <typename T>
__device__ __forceinline__ T plain_gradient(const T *q, uint32_t i, uint32_t st, unsigned m, float shift) {
    if ((m & 15u) == 15u) return ((T)8 * (q[i + st] - q[i - st]) - (q[i + 2 * st] - q[i - 2 * st])) * ((T)1 / (T)12);
    const bool below = (m & 1u) != 0, above = (m & 2u) != 0;
    const T c = q[i];
    T faces = 0, loops = 0;
    if (above) {
        faces += (T)0.5 * (q[i + st] - c);
        if (m & 8u) loops += q[i + st] - q[i + 2 * st];
    } else if (shift < 0.0f) {
        faces -= c;
    }
    if (below) {
        faces += (T)0.5 * (c - q[i - st]);
        if (m & 4u) loops += q[i - 2 * st] - q[i - st];
    } else if (shift > 0.0f) {
        faces += c;
    }
    if (below && above) loops += q[i + st] - q[i - st];
    return faces + loops * ((T)1 / (T)12);
}

// D(q) at a moving cell: the plain way (fdtd.hpp:1970-1974) or round the solids
// (fdtd.hpp:1978-1991 inside the moving air, fdtd.hpp:1996-2020 on its border).
template <typename T, bool ROUND>
__device__ __forceinline__ T moved(const Flow &f, const T *q, uint32_t i) {
    if (!ROUND) {
        const float sx = f.shift_x[i], sy = f.shift_y[i];
        const unsigned m = f.mask[i];
        return -((T)sx * plain_gradient(q, i, 1u, m & 15u, sx) + (T)sy * plain_gradient(q, i, f.sy, m >> 4, sy));
    }
    const bool border = f.mask[i] == 2;
    const T c = q[i];
    T sum = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const uint32_t st = d == 0 ? 1u : (d == 1 ? f.sy : f.sz);
        const float *w = f.wind[d], *l = f.loop[d];
        const T above = q[i + st], below = q[i - st];
        if (!border) {
            sum += (T)0.5 * ((T)w[i] * (above - c) + (T)w[i - st] * (c - below)) + (T)l[i] * (above - q[i + 2 * st]) +
                   (T)l[i - st] * (above - below) + (T)l[i - 2 * st] * (q[i - 2 * st] - below);
            continue;
        }
        if (f.mask[i + st]) {
            sum += (T)0.5 * (T)w[i] * (above - c);
        } else if (w[i] < 0.0f) {
            sum -= (T)w[i] * c;
        }
        if (f.mask[i - st]) {
            sum += (T)0.5 * (T)w[i - st] * (c - below);
        } else if (w[i - st] > 0.0f) {
            sum += (T)w[i - st] * c;
        }
        sum += (T)l[i] * (above - q[i + 2 * st]) + (T)l[i - st] * (above - below) + (T)l[i - 2 * st] * (q[i - 2 * st] - below);
    }
    return -sum;
}

// Stage STAGE (1, 2 or 3) of the carry, both levels: blockIdx.y 0 carries q0, 1 carries q1. The
// halo's entries (stages 1 and 2 only) copy the level into the stage buffer.
template <typename T, bool ROUND, int STAGE>
__global__ void __launch_bounds__(256) carry_kernel(Flow f, T *q0, T *q1) {
    T *q = blockIdx.y ? q1 : q0;
    T *t1 = static_cast<T *>(f.t1[blockIdx.y]), *t2 = static_cast<T *>(f.t2[blockIdx.y]);
    const uint32_t count = STAGE == 3 ? f.moving : f.count;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const uint32_t i = f.cells[e];
        if (e >= f.moving) {
            (STAGE == 1 ? t1 : t2)[i] = q[i];
            continue;
        }
        if (STAGE == 1) {
            t1[i] = q[i] + moved<T, ROUND>(f, q, i);
        } else if (STAGE == 2) {
            t2[i] = (T)0.75 * q[i] + (T)0.25 * (t1[i] + moved<T, ROUND>(f, t1, i));
        } else {
            q[i] = q[i] + ((T)2 / (T)3) * ((t2[i] + moved<T, ROUND>(f, t2, i)) - q[i]);
        }
    }
}

}  // namespace fdtd
