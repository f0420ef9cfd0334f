// Generated by gen_median_net.py (Batcher odd-even merge sort, pruned to the middle output).
#pragma once

namespace mr {
namespace ringalt {

// middle of 3 values: 4 min/max operations
__device__ __forceinline__ float median_net3(float (&v)[3])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    v[2] = fmaxf(v[0], v[2]);
    v[1] = fminf(v[1], v[2]);
    return v[1];
}

// middle of 5 values: 12 min/max operations
__device__ __forceinline__ float median_net5(float (&v)[5])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    { const float t = fminf(v[2], v[3]); v[3] = fmaxf(v[2], v[3]); v[2] = t; }
    { const float t = fminf(v[0], v[2]); v[2] = fmaxf(v[0], v[2]); v[0] = t; }
    v[1] = fminf(v[1], v[3]);
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    v[4] = fmaxf(v[0], v[4]);
    v[2] = fminf(v[2], v[4]);
    v[2] = fmaxf(v[1], v[2]);
    return v[2];
}

// middle of 9 values: 40 min/max operations
__device__ __forceinline__ float median_net9(float (&v)[9])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    { const float t = fminf(v[2], v[3]); v[3] = fmaxf(v[2], v[3]); v[2] = t; }
    { const float t = fminf(v[0], v[2]); v[2] = fmaxf(v[0], v[2]); v[0] = t; }
    { const float t = fminf(v[1], v[3]); v[3] = fmaxf(v[1], v[3]); v[1] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[4], v[5]); v[5] = fmaxf(v[4], v[5]); v[4] = t; }
    { const float t = fminf(v[6], v[7]); v[7] = fmaxf(v[6], v[7]); v[6] = t; }
    { const float t = fminf(v[4], v[6]); v[6] = fmaxf(v[4], v[6]); v[4] = t; }
    { const float t = fminf(v[5], v[7]); v[7] = fmaxf(v[5], v[7]); v[5] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[0], v[4]); v[4] = fmaxf(v[0], v[4]); v[0] = t; }
    { const float t = fminf(v[2], v[6]); v[6] = fmaxf(v[2], v[6]); v[2] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[1], v[5]); v[5] = fmaxf(v[1], v[5]); v[1] = t; }
    v[3] = fminf(v[3], v[7]);
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    v[2] = fmaxf(v[1], v[2]);
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    v[5] = fminf(v[5], v[6]);
    v[8] = fmaxf(v[0], v[8]);
    v[4] = fminf(v[4], v[8]);
    v[4] = fmaxf(v[2], v[4]);
    v[3] = fminf(v[3], v[5]);
    v[4] = fmaxf(v[3], v[4]);
    return v[4];
}

// middle of 11 values: 54 min/max operations
__device__ __forceinline__ float median_net11(float (&v)[11])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    { const float t = fminf(v[2], v[3]); v[3] = fmaxf(v[2], v[3]); v[2] = t; }
    { const float t = fminf(v[0], v[2]); v[2] = fmaxf(v[0], v[2]); v[0] = t; }
    { const float t = fminf(v[1], v[3]); v[3] = fmaxf(v[1], v[3]); v[1] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[4], v[5]); v[5] = fmaxf(v[4], v[5]); v[4] = t; }
    { const float t = fminf(v[6], v[7]); v[7] = fmaxf(v[6], v[7]); v[6] = t; }
    { const float t = fminf(v[4], v[6]); v[6] = fmaxf(v[4], v[6]); v[4] = t; }
    { const float t = fminf(v[5], v[7]); v[7] = fmaxf(v[5], v[7]); v[5] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[0], v[4]); v[4] = fmaxf(v[0], v[4]); v[0] = t; }
    { const float t = fminf(v[2], v[6]); v[6] = fmaxf(v[2], v[6]); v[2] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[1], v[5]); v[5] = fmaxf(v[1], v[5]); v[1] = t; }
    v[3] = fminf(v[3], v[7]);
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[8], v[9]); v[9] = fmaxf(v[8], v[9]); v[8] = t; }
    { const float t = fminf(v[8], v[10]); v[10] = fmaxf(v[8], v[10]); v[8] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    v[8] = fmaxf(v[0], v[8]);
    v[8] = fmaxf(v[4], v[8]);
    v[10] = fmaxf(v[2], v[10]);
    v[6] = fminf(v[6], v[10]);
    v[6] = fminf(v[6], v[8]);
    v[9] = fmaxf(v[1], v[9]);
    v[5] = fminf(v[5], v[9]);
    v[5] = fmaxf(v[3], v[5]);
    v[5] = fminf(v[5], v[6]);
    return v[5];
}

// middle of 15 values: 84 min/max operations
__device__ __forceinline__ float median_net15(float (&v)[15])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    { const float t = fminf(v[2], v[3]); v[3] = fmaxf(v[2], v[3]); v[2] = t; }
    { const float t = fminf(v[0], v[2]); v[2] = fmaxf(v[0], v[2]); v[0] = t; }
    { const float t = fminf(v[1], v[3]); v[3] = fmaxf(v[1], v[3]); v[1] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[4], v[5]); v[5] = fmaxf(v[4], v[5]); v[4] = t; }
    { const float t = fminf(v[6], v[7]); v[7] = fmaxf(v[6], v[7]); v[6] = t; }
    { const float t = fminf(v[4], v[6]); v[6] = fmaxf(v[4], v[6]); v[4] = t; }
    { const float t = fminf(v[5], v[7]); v[7] = fmaxf(v[5], v[7]); v[5] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[0], v[4]); v[4] = fmaxf(v[0], v[4]); v[0] = t; }
    { const float t = fminf(v[2], v[6]); v[6] = fmaxf(v[2], v[6]); v[2] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[1], v[5]); v[5] = fmaxf(v[1], v[5]); v[1] = t; }
    { const float t = fminf(v[3], v[7]); v[7] = fmaxf(v[3], v[7]); v[3] = t; }
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[8], v[9]); v[9] = fmaxf(v[8], v[9]); v[8] = t; }
    { const float t = fminf(v[10], v[11]); v[11] = fmaxf(v[10], v[11]); v[10] = t; }
    { const float t = fminf(v[8], v[10]); v[10] = fmaxf(v[8], v[10]); v[8] = t; }
    { const float t = fminf(v[9], v[11]); v[11] = fmaxf(v[9], v[11]); v[9] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[12], v[13]); v[13] = fmaxf(v[12], v[13]); v[12] = t; }
    { const float t = fminf(v[12], v[14]); v[14] = fmaxf(v[12], v[14]); v[12] = t; }
    { const float t = fminf(v[13], v[14]); v[14] = fmaxf(v[13], v[14]); v[13] = t; }
    { const float t = fminf(v[8], v[12]); v[12] = fmaxf(v[8], v[12]); v[8] = t; }
    { const float t = fminf(v[10], v[14]); v[14] = fmaxf(v[10], v[14]); v[10] = t; }
    { const float t = fminf(v[10], v[12]); v[12] = fmaxf(v[10], v[12]); v[10] = t; }
    { const float t = fminf(v[9], v[13]); v[13] = fmaxf(v[9], v[13]); v[9] = t; }
    { const float t = fminf(v[11], v[13]); v[13] = fmaxf(v[11], v[13]); v[11] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[11], v[12]); v[12] = fmaxf(v[11], v[12]); v[11] = t; }
    { const float t = fminf(v[13], v[14]); v[14] = fmaxf(v[13], v[14]); v[13] = t; }
    v[8] = fmaxf(v[0], v[8]);
    v[4] = fminf(v[4], v[12]);
    v[8] = fmaxf(v[4], v[8]);
    v[10] = fmaxf(v[2], v[10]);
    v[6] = fminf(v[6], v[14]);
    v[6] = fminf(v[6], v[10]);
    v[8] = fmaxf(v[6], v[8]);
    v[9] = fmaxf(v[1], v[9]);
    v[5] = fminf(v[5], v[13]);
    v[9] = fmaxf(v[5], v[9]);
    v[11] = fmaxf(v[3], v[11]);
    v[7] = fminf(v[7], v[11]);
    v[7] = fminf(v[7], v[9]);
    v[7] = fminf(v[7], v[8]);
    return v[7];
}

// middle of 25 values: 202 min/max operations
__device__ __forceinline__ float median_net25(float (&v)[25])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    { const float t = fminf(v[2], v[3]); v[3] = fmaxf(v[2], v[3]); v[2] = t; }
    { const float t = fminf(v[0], v[2]); v[2] = fmaxf(v[0], v[2]); v[0] = t; }
    { const float t = fminf(v[1], v[3]); v[3] = fmaxf(v[1], v[3]); v[1] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[4], v[5]); v[5] = fmaxf(v[4], v[5]); v[4] = t; }
    { const float t = fminf(v[6], v[7]); v[7] = fmaxf(v[6], v[7]); v[6] = t; }
    { const float t = fminf(v[4], v[6]); v[6] = fmaxf(v[4], v[6]); v[4] = t; }
    { const float t = fminf(v[5], v[7]); v[7] = fmaxf(v[5], v[7]); v[5] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[0], v[4]); v[4] = fmaxf(v[0], v[4]); v[0] = t; }
    { const float t = fminf(v[2], v[6]); v[6] = fmaxf(v[2], v[6]); v[2] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[1], v[5]); v[5] = fmaxf(v[1], v[5]); v[1] = t; }
    { const float t = fminf(v[3], v[7]); v[7] = fmaxf(v[3], v[7]); v[3] = t; }
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[8], v[9]); v[9] = fmaxf(v[8], v[9]); v[8] = t; }
    { const float t = fminf(v[10], v[11]); v[11] = fmaxf(v[10], v[11]); v[10] = t; }
    { const float t = fminf(v[8], v[10]); v[10] = fmaxf(v[8], v[10]); v[8] = t; }
    { const float t = fminf(v[9], v[11]); v[11] = fmaxf(v[9], v[11]); v[9] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[12], v[13]); v[13] = fmaxf(v[12], v[13]); v[12] = t; }
    { const float t = fminf(v[14], v[15]); v[15] = fmaxf(v[14], v[15]); v[14] = t; }
    { const float t = fminf(v[12], v[14]); v[14] = fmaxf(v[12], v[14]); v[12] = t; }
    { const float t = fminf(v[13], v[15]); v[15] = fmaxf(v[13], v[15]); v[13] = t; }
    { const float t = fminf(v[13], v[14]); v[14] = fmaxf(v[13], v[14]); v[13] = t; }
    { const float t = fminf(v[8], v[12]); v[12] = fmaxf(v[8], v[12]); v[8] = t; }
    { const float t = fminf(v[10], v[14]); v[14] = fmaxf(v[10], v[14]); v[10] = t; }
    { const float t = fminf(v[10], v[12]); v[12] = fmaxf(v[10], v[12]); v[10] = t; }
    { const float t = fminf(v[9], v[13]); v[13] = fmaxf(v[9], v[13]); v[9] = t; }
    { const float t = fminf(v[11], v[15]); v[15] = fmaxf(v[11], v[15]); v[11] = t; }
    { const float t = fminf(v[11], v[13]); v[13] = fmaxf(v[11], v[13]); v[11] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[11], v[12]); v[12] = fmaxf(v[11], v[12]); v[11] = t; }
    { const float t = fminf(v[13], v[14]); v[14] = fmaxf(v[13], v[14]); v[13] = t; }
    { const float t = fminf(v[0], v[8]); v[8] = fmaxf(v[0], v[8]); v[0] = t; }
    { const float t = fminf(v[4], v[12]); v[12] = fmaxf(v[4], v[12]); v[4] = t; }
    { const float t = fminf(v[4], v[8]); v[8] = fmaxf(v[4], v[8]); v[4] = t; }
    { const float t = fminf(v[2], v[10]); v[10] = fmaxf(v[2], v[10]); v[2] = t; }
    { const float t = fminf(v[6], v[14]); v[14] = fmaxf(v[6], v[14]); v[6] = t; }
    { const float t = fminf(v[6], v[10]); v[10] = fmaxf(v[6], v[10]); v[6] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[6], v[8]); v[8] = fmaxf(v[6], v[8]); v[6] = t; }
    { const float t = fminf(v[10], v[12]); v[12] = fmaxf(v[10], v[12]); v[10] = t; }
    { const float t = fminf(v[1], v[9]); v[9] = fmaxf(v[1], v[9]); v[1] = t; }
    { const float t = fminf(v[5], v[13]); v[13] = fmaxf(v[5], v[13]); v[5] = t; }
    { const float t = fminf(v[5], v[9]); v[9] = fmaxf(v[5], v[9]); v[5] = t; }
    { const float t = fminf(v[3], v[11]); v[11] = fmaxf(v[3], v[11]); v[3] = t; }
    v[7] = fminf(v[7], v[15]);
    { const float t = fminf(v[7], v[11]); v[11] = fmaxf(v[7], v[11]); v[7] = t; }
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    { const float t = fminf(v[7], v[9]); v[9] = fmaxf(v[7], v[9]); v[7] = t; }
    { const float t = fminf(v[11], v[13]); v[13] = fmaxf(v[11], v[13]); v[11] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[7], v[8]); v[8] = fmaxf(v[7], v[8]); v[7] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[11], v[12]); v[12] = fmaxf(v[11], v[12]); v[11] = t; }
    v[13] = fminf(v[13], v[14]);
    { const float t = fminf(v[16], v[17]); v[17] = fmaxf(v[16], v[17]); v[16] = t; }
    { const float t = fminf(v[18], v[19]); v[19] = fmaxf(v[18], v[19]); v[18] = t; }
    { const float t = fminf(v[16], v[18]); v[18] = fmaxf(v[16], v[18]); v[16] = t; }
    { const float t = fminf(v[17], v[19]); v[19] = fmaxf(v[17], v[19]); v[17] = t; }
    { const float t = fminf(v[17], v[18]); v[18] = fmaxf(v[17], v[18]); v[17] = t; }
    { const float t = fminf(v[20], v[21]); v[21] = fmaxf(v[20], v[21]); v[20] = t; }
    { const float t = fminf(v[22], v[23]); v[23] = fmaxf(v[22], v[23]); v[22] = t; }
    { const float t = fminf(v[20], v[22]); v[22] = fmaxf(v[20], v[22]); v[20] = t; }
    { const float t = fminf(v[21], v[23]); v[23] = fmaxf(v[21], v[23]); v[21] = t; }
    { const float t = fminf(v[21], v[22]); v[22] = fmaxf(v[21], v[22]); v[21] = t; }
    { const float t = fminf(v[16], v[20]); v[20] = fmaxf(v[16], v[20]); v[16] = t; }
    { const float t = fminf(v[18], v[22]); v[22] = fmaxf(v[18], v[22]); v[18] = t; }
    { const float t = fminf(v[18], v[20]); v[20] = fmaxf(v[18], v[20]); v[18] = t; }
    { const float t = fminf(v[17], v[21]); v[21] = fmaxf(v[17], v[21]); v[17] = t; }
    { const float t = fminf(v[19], v[23]); v[23] = fmaxf(v[19], v[23]); v[19] = t; }
    { const float t = fminf(v[19], v[21]); v[21] = fmaxf(v[19], v[21]); v[19] = t; }
    { const float t = fminf(v[17], v[18]); v[18] = fmaxf(v[17], v[18]); v[17] = t; }
    { const float t = fminf(v[19], v[20]); v[20] = fmaxf(v[19], v[20]); v[19] = t; }
    { const float t = fminf(v[21], v[22]); v[22] = fmaxf(v[21], v[22]); v[21] = t; }
    { const float t = fminf(v[16], v[24]); v[24] = fmaxf(v[16], v[24]); v[16] = t; }
    { const float t = fminf(v[20], v[24]); v[24] = fmaxf(v[20], v[24]); v[20] = t; }
    { const float t = fminf(v[18], v[20]); v[20] = fmaxf(v[18], v[20]); v[18] = t; }
    { const float t = fminf(v[22], v[24]); v[24] = fmaxf(v[22], v[24]); v[22] = t; }
    { const float t = fminf(v[19], v[21]); v[21] = fmaxf(v[19], v[21]); v[19] = t; }
    { const float t = fminf(v[17], v[18]); v[18] = fmaxf(v[17], v[18]); v[17] = t; }
    { const float t = fminf(v[19], v[20]); v[20] = fmaxf(v[19], v[20]); v[19] = t; }
    { const float t = fminf(v[21], v[22]); v[22] = fmaxf(v[21], v[22]); v[21] = t; }
    { const float t = fminf(v[23], v[24]); v[24] = fmaxf(v[23], v[24]); v[23] = t; }
    v[16] = fmaxf(v[0], v[16]);
    v[8] = fminf(v[8], v[24]);
    v[16] = fmaxf(v[8], v[16]);
    v[20] = fmaxf(v[4], v[20]);
    v[12] = fminf(v[12], v[20]);
    v[12] = fminf(v[12], v[16]);
    v[18] = fmaxf(v[2], v[18]);
    v[10] = fminf(v[10], v[18]);
    v[6] = fminf(v[6], v[22]);
    v[10] = fmaxf(v[6], v[10]);
    v[12] = fmaxf(v[10], v[12]);
    v[17] = fmaxf(v[1], v[17]);
    v[17] = fmaxf(v[9], v[17]);
    v[21] = fmaxf(v[5], v[21]);
    v[13] = fminf(v[13], v[21]);
    v[13] = fminf(v[13], v[17]);
    v[19] = fmaxf(v[3], v[19]);
    v[11] = fminf(v[11], v[19]);
    v[7] = fminf(v[7], v[23]);
    v[11] = fmaxf(v[7], v[11]);
    v[11] = fminf(v[11], v[13]);
    v[12] = fmaxf(v[11], v[12]);
    return v[12];
}

// ranks 7..12 (0-based) of 20 values into v[7..12]: 168 min/max operations
__device__ __forceinline__ void rank_net20_7_12(float (&v)[20])
{
    { const float t = fminf(v[0], v[1]); v[1] = fmaxf(v[0], v[1]); v[0] = t; }
    { const float t = fminf(v[2], v[3]); v[3] = fmaxf(v[2], v[3]); v[2] = t; }
    { const float t = fminf(v[0], v[2]); v[2] = fmaxf(v[0], v[2]); v[0] = t; }
    { const float t = fminf(v[1], v[3]); v[3] = fmaxf(v[1], v[3]); v[1] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[4], v[5]); v[5] = fmaxf(v[4], v[5]); v[4] = t; }
    { const float t = fminf(v[6], v[7]); v[7] = fmaxf(v[6], v[7]); v[6] = t; }
    { const float t = fminf(v[4], v[6]); v[6] = fmaxf(v[4], v[6]); v[4] = t; }
    { const float t = fminf(v[5], v[7]); v[7] = fmaxf(v[5], v[7]); v[5] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[0], v[4]); v[4] = fmaxf(v[0], v[4]); v[0] = t; }
    { const float t = fminf(v[2], v[6]); v[6] = fmaxf(v[2], v[6]); v[2] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[1], v[5]); v[5] = fmaxf(v[1], v[5]); v[1] = t; }
    { const float t = fminf(v[3], v[7]); v[7] = fmaxf(v[3], v[7]); v[3] = t; }
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[8], v[9]); v[9] = fmaxf(v[8], v[9]); v[8] = t; }
    { const float t = fminf(v[10], v[11]); v[11] = fmaxf(v[10], v[11]); v[10] = t; }
    { const float t = fminf(v[8], v[10]); v[10] = fmaxf(v[8], v[10]); v[8] = t; }
    { const float t = fminf(v[9], v[11]); v[11] = fmaxf(v[9], v[11]); v[9] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[12], v[13]); v[13] = fmaxf(v[12], v[13]); v[12] = t; }
    { const float t = fminf(v[14], v[15]); v[15] = fmaxf(v[14], v[15]); v[14] = t; }
    { const float t = fminf(v[12], v[14]); v[14] = fmaxf(v[12], v[14]); v[12] = t; }
    { const float t = fminf(v[13], v[15]); v[15] = fmaxf(v[13], v[15]); v[13] = t; }
    { const float t = fminf(v[13], v[14]); v[14] = fmaxf(v[13], v[14]); v[13] = t; }
    { const float t = fminf(v[8], v[12]); v[12] = fmaxf(v[8], v[12]); v[8] = t; }
    { const float t = fminf(v[10], v[14]); v[14] = fmaxf(v[10], v[14]); v[10] = t; }
    { const float t = fminf(v[10], v[12]); v[12] = fmaxf(v[10], v[12]); v[10] = t; }
    { const float t = fminf(v[9], v[13]); v[13] = fmaxf(v[9], v[13]); v[9] = t; }
    { const float t = fminf(v[11], v[15]); v[15] = fmaxf(v[11], v[15]); v[11] = t; }
    { const float t = fminf(v[11], v[13]); v[13] = fmaxf(v[11], v[13]); v[11] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[11], v[12]); v[12] = fmaxf(v[11], v[12]); v[11] = t; }
    { const float t = fminf(v[13], v[14]); v[14] = fmaxf(v[13], v[14]); v[13] = t; }
    { const float t = fminf(v[0], v[8]); v[8] = fmaxf(v[0], v[8]); v[0] = t; }
    { const float t = fminf(v[4], v[12]); v[12] = fmaxf(v[4], v[12]); v[4] = t; }
    { const float t = fminf(v[4], v[8]); v[8] = fmaxf(v[4], v[8]); v[4] = t; }
    { const float t = fminf(v[2], v[10]); v[10] = fmaxf(v[2], v[10]); v[2] = t; }
    { const float t = fminf(v[6], v[14]); v[14] = fmaxf(v[6], v[14]); v[6] = t; }
    { const float t = fminf(v[6], v[10]); v[10] = fmaxf(v[6], v[10]); v[6] = t; }
    { const float t = fminf(v[2], v[4]); v[4] = fmaxf(v[2], v[4]); v[2] = t; }
    { const float t = fminf(v[6], v[8]); v[8] = fmaxf(v[6], v[8]); v[6] = t; }
    { const float t = fminf(v[10], v[12]); v[12] = fmaxf(v[10], v[12]); v[10] = t; }
    { const float t = fminf(v[1], v[9]); v[9] = fmaxf(v[1], v[9]); v[1] = t; }
    { const float t = fminf(v[5], v[13]); v[13] = fmaxf(v[5], v[13]); v[5] = t; }
    { const float t = fminf(v[5], v[9]); v[9] = fmaxf(v[5], v[9]); v[5] = t; }
    { const float t = fminf(v[3], v[11]); v[11] = fmaxf(v[3], v[11]); v[3] = t; }
    v[7] = fminf(v[7], v[15]);
    { const float t = fminf(v[7], v[11]); v[11] = fmaxf(v[7], v[11]); v[7] = t; }
    { const float t = fminf(v[3], v[5]); v[5] = fmaxf(v[3], v[5]); v[3] = t; }
    { const float t = fminf(v[7], v[9]); v[9] = fmaxf(v[7], v[9]); v[7] = t; }
    { const float t = fminf(v[11], v[13]); v[13] = fmaxf(v[11], v[13]); v[11] = t; }
    { const float t = fminf(v[1], v[2]); v[2] = fmaxf(v[1], v[2]); v[1] = t; }
    { const float t = fminf(v[3], v[4]); v[4] = fmaxf(v[3], v[4]); v[3] = t; }
    { const float t = fminf(v[5], v[6]); v[6] = fmaxf(v[5], v[6]); v[5] = t; }
    { const float t = fminf(v[7], v[8]); v[8] = fmaxf(v[7], v[8]); v[7] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[11], v[12]); v[12] = fmaxf(v[11], v[12]); v[11] = t; }
    v[13] = fminf(v[13], v[14]);
    { const float t = fminf(v[16], v[17]); v[17] = fmaxf(v[16], v[17]); v[16] = t; }
    { const float t = fminf(v[18], v[19]); v[19] = fmaxf(v[18], v[19]); v[18] = t; }
    { const float t = fminf(v[16], v[18]); v[18] = fmaxf(v[16], v[18]); v[16] = t; }
    { const float t = fminf(v[17], v[19]); v[19] = fmaxf(v[17], v[19]); v[17] = t; }
    { const float t = fminf(v[17], v[18]); v[18] = fmaxf(v[17], v[18]); v[17] = t; }
    { const float t = fminf(v[17], v[18]); v[18] = fmaxf(v[17], v[18]); v[17] = t; }
    { const float t = fminf(v[17], v[18]); v[18] = fmaxf(v[17], v[18]); v[17] = t; }
    v[16] = fmaxf(v[0], v[16]);
    { const float t = fminf(v[8], v[16]); v[16] = fmaxf(v[8], v[16]); v[8] = t; }
    v[8] = fmaxf(v[4], v[8]);
    v[12] = fminf(v[12], v[16]);
    v[18] = fmaxf(v[2], v[18]);
    v[10] = fminf(v[10], v[18]);
    { const float t = fminf(v[6], v[10]); v[10] = fmaxf(v[6], v[10]); v[6] = t; }
    v[8] = fmaxf(v[6], v[8]);
    { const float t = fminf(v[10], v[12]); v[12] = fmaxf(v[10], v[12]); v[10] = t; }
    v[17] = fmaxf(v[1], v[17]);
    { const float t = fminf(v[9], v[17]); v[17] = fmaxf(v[9], v[17]); v[9] = t; }
    v[9] = fmaxf(v[5], v[9]);
    v[13] = fminf(v[13], v[17]);
    v[19] = fmaxf(v[3], v[19]);
    v[11] = fminf(v[11], v[19]);
    { const float t = fminf(v[7], v[11]); v[11] = fmaxf(v[7], v[11]); v[7] = t; }
    { const float t = fminf(v[7], v[9]); v[9] = fmaxf(v[7], v[9]); v[7] = t; }
    v[11] = fminf(v[11], v[13]);
    { const float t = fminf(v[7], v[8]); v[8] = fmaxf(v[7], v[8]); v[7] = t; }
    { const float t = fminf(v[9], v[10]); v[10] = fmaxf(v[9], v[10]); v[9] = t; }
    { const float t = fminf(v[11], v[12]); v[12] = fmaxf(v[11], v[12]); v[11] = t; }
}

} // namespace ringalt
} // namespace mr
