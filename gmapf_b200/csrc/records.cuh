// records.cuh -- one 32-byte access per search record (device code only).
//
// A record (`Rec`, internal.h) is one 32-byte L2 sector.  Reading or writing
// it with a single 256-bit access costs one L1 pass instead of two, and a
// whole-sector store lets L2 evict the sector without first filling the
// other half from DRAM.  Records are 32-byte aligned: every record array
// starts at an allocation (or array) boundary and holds whole records.
#pragma once

#include "internal.h"

namespace gmapf_b200 {

// the whole record, through L2 (records are written by other threads of the warp)
__device__ __forceinline__ void ld_rec(const Rec* r, int4& a, int4& b) {
    asm volatile("ld.global.cg.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
                 : "l"(r));
}

// {stamp or jump ancestor, G<<1|dir, ancestors 1..6}
__device__ __forceinline__ void st_rec(Rec* r, unsigned stamp, int gd, int a0, int a1, int a2, int a3, int a4,
                                       int a5) {
    asm volatile("st.global.cg.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(r), "r"((int)stamp), "r"(gd),
                 "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(a4), "r"(a5)
                 : "memory");
}

}  // namespace gmapf_b200
