// Cartesian bookkeeping for the table-driven kernels (generic, coop).
//
// Every Cartesian Gaussian of AM level 0..CI_MAXL gets a flat index
// (levels in order, Psi4 order inside a level).  For each one the table
// holds its exponents, level, Psi4 position, the recursion direction of the
// reference planner (smallest non-zero exponent, right-most on ties:
// generator/ostei/Makowski.hpp:113-117, the same rule as the reference's
// recur_lookup table, python/gen_recurinfo.py) and the flat indices of its
// neighbours g-1_x, g-2_dir, g+1_x (-1 when they do not exist).
//
// The table is file-static: each translation unit that includes this
// header owns a copy in constant memory and uploads it with
// upload_cart_info() before its first launch on a device.
#pragma once

#include <cuda_runtime.h>
#include <array>
#include <mutex>
#include <vector>

#include "simint_b200.h"

#define CI_MAXL 10
#define CI_NCART 286               // flat indices of levels 0..CI_MAXL

struct CartInfo
{
    signed char ijk[3];
    signed char lev, pos, dir;
    short m1[3];
    short m2;
    short p1[3];
};

static __constant__ CartInfo c_cartinfo[CI_NCART];

__device__ __forceinline__ int cart_index_dev(int g, int ordering)
{
    const CartInfo & c = c_cartinfo[g];
    const int l = c.lev;
    if(ordering == SIMINT_B200_ORDERING_GAMESS && (l == 2 || l == 3))
    {
        // generator/Ordering_GAMESS.cpp:20-41
        const int i = c.ijk[0], j = c.ijk[1], k = c.ijk[2];
        if(l == 2)
        {
            if(i == 2) return 0;
            if(j == 2) return 1;
            if(k == 2) return 2;
            if(i == 1 && j == 1) return 3;
            if(i == 1) return 4;
            return 5;
        }
        if(i == 3) return 0;
        if(j == 3) return 1;
        if(k == 3) return 2;
        if(i == 2 && j == 1) return 3;
        if(i == 2) return 4;
        if(i == 1 && j == 2) return 5;
        if(j == 2) return 6;
        if(i == 1 && k == 2) return 7;
        if(k == 2) return 8;
        return 9;
    }
    return c.pos;
}

static inline int ci_lev_off(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }

static inline int ci_flat(int i, int j, int k)
{
    if(i < 0 || j < 0 || k < 0)
        return -1;
    const int l = i + j + k;
    if(l > CI_MAXL)
        return -1;
    return ci_lev_off(l) + ((l - i) * (l - i + 1)) / 2 + k;
}

// Fill t[0 .. CI_NCART) with the table (no allocation).
static void cart_table_fill(CartInfo * t)
{
    for(int l = 0; l <= CI_MAXL; l++)
    {
        int p = 0;
        for(int i = l; i >= 0; i--)
            for(int j = l - i; j >= 0; j--, p++)
            {
                const int k = l - i - j;
                CartInfo & c = t[ci_lev_off(l) + p];
                c.ijk[0] = (signed char)i; c.ijk[1] = (signed char)j; c.ijk[2] = (signed char)k;
                c.lev = (signed char)l;
                c.pos = (signed char)p;
                const int e[3] = {i, j, k};
                int mn = 1000, dir = -1;
                for(int x = 0; x < 3; x++)
                    if(e[x] > 0 && e[x] < mn) mn = e[x];
                for(int x = 2; x >= 0; x--)
                    if(e[x] == mn) { dir = x; break; }
                c.dir = (signed char)dir;
                c.m1[0] = (short)ci_flat(i - 1, j, k);
                c.m1[1] = (short)ci_flat(i, j - 1, k);
                c.m1[2] = (short)ci_flat(i, j, k - 1);
                c.p1[0] = (short)ci_flat(i + 1, j, k);
                c.p1[1] = (short)ci_flat(i, j + 1, k);
                c.p1[2] = (short)ci_flat(i, j, k + 1);
                int q[3] = {i, j, k};
                if(dir >= 0) q[dir] -= 2;
                c.m2 = (short)(dir >= 0 ? ci_flat(q[0], q[1], q[2]) : -1);
            }
    }
}

// The table on the host (the same contents the device copy gets).
static std::vector<CartInfo> cart_table_host()
{
    std::vector<CartInfo> t(CI_NCART);
    cart_table_fill(t.data());
    return t;
}

// Once per device, under a lock: calls from several host threads may come
// first at the same time.
static void upload_cart_info()
{
    static std::mutex m;
    static std::vector<char> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(m);
    if((int)done.size() > dev && done[dev])
        return;
    const std::vector<CartInfo> t = cart_table_host();
    cudaMemcpyToSymbol(c_cartinfo, t.data(), sizeof(CartInfo) * CI_NCART);
    if((int)done.size() <= dev)
        done.resize(dev + 1, 0);
    done[dev] = 1;
}
