// bc.cuh: the BC4 block arithmetic shared by the device refinement (refine.cu) and the host asset writer (asset.cpp):
// the palette a decoder evaluates from two endpoints, and the seed pack of one block of one channel.
#pragma once

#include <cmath>
#include <cstdint>

#include "common.cuh"

namespace nb
{

// The palette as a decoder evaluates it (shared/bc_pack.h:62-77), both modes.
__host__ __device__ __forceinline__ void bc4_palette(int r0, int r1, float p[8])
{
    p[0] = (float)r0;
    p[1] = (float)r1;
    if (r0 > r1)
    {
        for (int i = 2; i < 8; i++)
            p[i] = (float)((8 - i) * r0 + (i - 1) * r1) / 7.0f;
    }
    else
    {
        for (int i = 2; i < 6; i++)
            p[i] = (float)((6 - i) * r0 + (i - 1) * r1) / 5.0f;
        p[6] = 0.0f;
        p[7] = 255.0f;
    }
}

// One block of one channel (shared/bc_pack.h:95-166): sixteen stored bytes at `bits` bits, edge-clamped by the
// caller, to endpoints and selectors.
__host__ __device__ inline void bc4_seed_block(const uint8_t v[16], int bits, int& r0, int& r1, uint8_t sel[16])
{
    if (bits <= 3)
    {
        if (bits == 3)
        {
            r0 = 255;
            r1 = 0;
            for (int t = 0; t < 16; t++)
            {
                const int k = v[t] >> 5;
                sel[t] = (uint8_t)(k == 7 ? 0 : (k == 0 ? 1 : 8 - k));
            }
        }
        else if (bits == 2)
        {
            r0 = 85;
            r1 = 170;
            for (int t = 0; t < 16; t++)
            {
                const int k = v[t] >> 6;
                sel[t] = (uint8_t)(k == 0 ? 6 : (k == 1 ? 0 : (k == 2 ? 1 : 7)));
            }
        }
        else
        {
            r0 = 0;
            r1 = 255;
            for (int t = 0; t < 16; t++)
                sel[t] = (uint8_t)((v[t] >> 7) ? 7 : 6);
        }
        return;
    }
    const int levels = (1 << bits) - 1;
    int kmin = levels, kmax = 0;
    for (int t = 0; t < 16; t++)
    {
        const int k = v[t] >> (8 - bits);
        kmin = k < kmin ? k : kmin;
        kmax = k > kmax ? k : kmax;
    }
    r0 = (int)llround(kmax * 255.0 / levels);
    r1 = (int)llround(kmin * 255.0 / levels);
    if (r0 == r1)
    {
        for (int t = 0; t < 16; t++)
            sel[t] = 0;
        return;
    }
    float p[8];
    bc4_palette(r0, r1, p);
    for (int t = 0; t < 16; t++)
    {
        const float target = (float)(v[t] >> (8 - bits)) * 255.0f / (float)levels;
        int best = 0;
        float best_d = 1e30f;
        for (int i = 0; i < 8; i++)
        {
            const float d = fabsf(p[i] - target);
            if (d < best_d)
            {
                best_d = d;
                best = i;
            }
        }
        sel[t] = (uint8_t)best;
    }
}

}   // namespace nb
