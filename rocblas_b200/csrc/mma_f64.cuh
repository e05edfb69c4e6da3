// The FP64 tensor instructions of B200 (mma.sync .f64; the tcgen05 tensor cores have no f64
// kind), shared by the GEMM tiles, the chain solve and the block solve's updates.
#pragma once

namespace rb200
{

// mma.sync m16n8k8 .f64 (sm_90+ shape; 1024 FMAs per instruction).  Fragments, with
// g = lane / 4 and t = lane % 4: A (16x8): a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4);
// B (8x8): b0 (t, g), b1 (t+4, g); C (16x8): c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1).
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
                 "{%8,%9}, {%0,%1,%2,%3};\n"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// mma.sync m16n8k16 .f64: the k8 fragments of two consecutive k8 steps side by side,
// a_{2q+r} = A(g + 8r, t + 4q), b_q = B(t + 4q, g) for q = 0..3, r = 0..1.
__device__ __forceinline__ void dmma_16x8x16(double (&d)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                 "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
                   "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

} // namespace rb200
