/* Cell arithmetic shared by the device index builders (index_gpu.cu) and the MortonGrid
 * (morton.cu): the cell of a point and the box of a Morton cell, in the reference builders' float
 * expressions (IEEE single subtract, divide and multiply, no contraction, truncation toward
 * zero), so that every cell and node box equals the host builder's bit for bit. */
#pragma once

#include <cstdint>

namespace gat {

struct CellParams {
    float rxmin, rymax, cell;
    int morton; /* 1: Grid (Morton id on an axis x axis grid), 0: FSG (row-major nx x ny) */
    int axis, nx, ny, vparam;
};

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
    v &= 0xFFFF;
    v = (v | (v << 8)) & 0x00FF00FF;
    v = (v | (v << 4)) & 0x0F0F0F0F;
    v = (v | (v << 2)) & 0x33333333;
    v = (v | (v << 1)) & 0x55555555;
    return v;
}
__device__ __forceinline__ uint32_t compact_bits(uint32_t v) {
    v &= 0x55555555;
    v = (v | (v >> 1)) & 0x33333333;
    v = (v | (v >> 2)) & 0x0F0F0F0F;
    v = (v | (v >> 4)) & 0x00FF00FF;
    v = (v | (v >> 8)) & 0x0000FFFF;
    return v;
}

/* float -> int truncation as the host's (int) cast gives it for every value that can land in a
 * grid; NaN and values beyond the int range are reported as outside (the host's conversion of
 * those yields INT_MIN, a negative row or column, hence also outside) */
__device__ __forceinline__ bool trunc_int(float v, int* out) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return false;
    *out = __float2int_rz(v);
    return true;
}

/* Grid::WhichCellPointIn (Grid.cpp:202-208) / FSG::WhichCellPointIn (FSG.cpp:88-93); -1 outside */
__device__ __forceinline__ int point_cell(const CellParams& p, float lon, float lat) {
    int row, col;
    if (!trunc_int(__fdiv_rn(__fsub_rn(p.rymax, lat), p.cell), &row)) return -1;
    if (!trunc_int(__fdiv_rn(__fsub_rn(lon, p.rxmin), p.cell), &col)) return -1;
    if (p.morton) {
        if (row < 0 || col < 0 || row >= p.axis || col >= p.axis) return -1;
        return (int)(spread_bits((uint32_t)col) | (spread_bits((uint32_t)row) << 1));
    }
    if (row < 0 || col < 0 || row >= p.ny || col >= p.nx) return -1;
    return row * p.nx + col;
}

/* the Morton cell's box (Grid.cpp:121): column from the even bits, row from the odd bits */
__device__ __forceinline__ float4 morton_cell_box(float rxmin, float rymax, float cell, int c) {
    const int col = (int)compact_bits((uint32_t)c), row = (int)compact_bits((uint32_t)c >> 1);
    return make_float4(__fadd_rn(rxmin, __fmul_rn(cell, (float)col)), __fsub_rn(rymax, __fmul_rn(cell, (float)(row + 1))),
                       __fadd_rn(rxmin, __fmul_rn(cell, (float)(col + 1))), __fsub_rn(rymax, __fmul_rn(cell, (float)row)));
}

}  // namespace gat
