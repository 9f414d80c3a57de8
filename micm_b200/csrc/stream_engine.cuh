// stream_engine.cuh -- the consumer side of the streamed schedule: one
// warp walks the segments of a block in shared memory (format in
// mechanism.hpp, StreamProgram) and applies them to its cell's working set.
//
// Every operand and target is a 16-bit byte offset from its array, so an
// address costs one mask or shift and one add.  Everything here is inlined
// into the kernel, where the arrays are known to live in shared memory.
#pragma once

#include "mechanism.hpp"

#include <cstdint>

namespace micmb
{
  namespace stream
  {
    __host__ __device__ inline int32_t Pad16(int32_t v)
    {
      return (v + 15) & ~15;
    }

    __device__ __forceinline__ double at(const double* base, uint32_t byte_offset)
    {
      return *reinterpret_cast<const double*>(reinterpret_cast<const char*>(base) + byte_offset);
    }

    __device__ __forceinline__ double& at(double* base, uint32_t byte_offset)
    {
      return *reinterpret_cast<double*>(reinterpret_cast<char*>(base) + byte_offset);
    }

    __device__ __forceinline__ double lo_op(const double* X, uint32_t q)
    {
      return at(X, q & 0xFFFFu);
    }

    __device__ __forceinline__ double hi_op(const double* Y, uint32_t q)
    {
      return at(Y, q >> 16);
    }

    enum
    {
      kGather = 0,
      kLU = 1,
      kSolve = 2,     // unit diagonal (L y = b)
      kSolveDiv = 3,  // divides by the diagonal (U x = y)
    };

    // value an item's finalisation needs besides its sum (read before the sum
    // is done).  The item's high half: LU: pivot row k of an L entry (< 0x8000),
    // 0x8000 | j for a diagonal, 0xFFFF / 0xFFFE for U entries / partial sums;
    // kSolveDiv: element index of the diagonal, or 0xFFFE / 0xFFFF.
    template<int KIND>
    __device__ __forceinline__ double fin_operand(uint32_t it, const double* X, const double* inv)
    {
      const uint32_t hi = it >> 16;
      if (KIND == kLU && hi < 0x8000u)
        return inv[hi];
      if (KIND == kSolveDiv && hi < 0xFFFEu)
        return X[hi];
      return 1.0;
    }

    // Per kind (x * 1.0 and x / 1.0 are exact, and a gather sum is never -0,
    // so the unflagged cases need no branch):
    //   kGather: out[e] = sum (+ alpha when the item is a diagonal), X = rates, Y = coefficients
    //   kLU:     in-place Crout update of A = X = Y = out: L entries sum * (1/a_kk), U entries
    //            and partial sums sum * 1, diagonals (kSegRecip segments) the sum and 1/sum
    //   kSolve / kSolveDiv: x_e = (x_e - sum A[a] x[b]) [/ A[aux]], X = A, Y = out = x
    template<int KIND>
    __device__ __forceinline__ void finalize(uint32_t it, double acc, double fin, double* out, double* inv,
                                             double alpha, int32_t flags)
    {
      const uint32_t e = it & 0xFFFFu, hi = it >> 16;
      if constexpr (KIND == kGather)
        at(out, e) = acc + ((hi != 0xFFFFu) ? alpha : 0.0);
      else if constexpr (KIND == kLU)
      {
        if (flags & kSegRecip)
        {
          at(out, e) = acc;
          inv[hi & 0x7FFFu] = 1.0 / acc;
        }
        else
          at(out, e) = acc * fin;
      }
      else if constexpr (KIND == kSolve)
        at(out, e) = acc;
      else
        at(out, e) = acc / fin;
    }

    template<int KIND>
    __device__ __forceinline__ double init_value(uint32_t it, const double* out)
    {
      return (KIND == kGather) ? 0.0 : at(out, it & 0xFFFFu);
    }

    // acc - sum over this lane's T terms of X[a] * Y[b], in term order.  Terms
    // come four to a uint4 (group g of this lane at tq[g * n]); the operands
    // of group g are loaded while the adds of group g - 1 run, and the
    // operand words one group further ahead.
    __device__ __forceinline__ double seg_chain(const uint4* tq, int32_t n, int32_t T, const double* X,
                                                const double* Yv, double acc)
    {
      if (T <= 0)
        return acc;
      const int32_t G = (T + 3) >> 2;
      const uint4 qa = tq[0];
      uint4 qb = (G > 1) ? tq[n] : qa;
      double a0 = lo_op(X, qa.x), b0 = hi_op(Yv, qa.x);
      double a1 = lo_op(X, qa.y), b1 = hi_op(Yv, qa.y);
      double a2 = lo_op(X, qa.z), b2 = hi_op(Yv, qa.z);
      double a3 = lo_op(X, qa.w), b3 = hi_op(Yv, qa.w);
      for (int32_t g = 1; g < G; ++g)
      {
        const uint4 qc = (g + 1 < G) ? tq[(g + 1) * n] : qb;
        const double c0 = lo_op(X, qb.x), d0 = hi_op(Yv, qb.x);
        const double c1 = lo_op(X, qb.y), d1 = hi_op(Yv, qb.y);
        const double c2 = lo_op(X, qb.z), d2 = hi_op(Yv, qb.z);
        const double c3 = lo_op(X, qb.w), d3 = hi_op(Yv, qb.w);
        acc -= a0 * b0;
        acc -= a1 * b1;
        acc -= a2 * b2;
        acc -= a3 * b3;
        a0 = c0;
        b0 = d0;
        a1 = c1;
        b1 = d1;
        a2 = c2;
        b2 = d2;
        a3 = c3;
        b3 = d3;
        qb = qc;
      }
      const int32_t rem = T - 4 * (G - 1);
      acc -= a0 * b0;
      if (rem > 1)
        acc -= a1 * b1;
      if (rem > 2)
        acc -= a2 * b2;
      if (rem > 3)
        acc -= a3 * b3;
      return acc;
    }

    // four independent sums per lane: term t of this lane's items at tq[t * n]
    __device__ __forceinline__ void seg_chain4(const uint4* tq, int32_t n, int32_t T, const double* X,
                                               const double* Yv, double (&acc)[4])
    {
      if (T <= 0)
        return;
      const uint4 q = tq[0];
      uint4 qn = (T > 1) ? tq[n] : q;
      double x0 = lo_op(X, q.x), y0 = hi_op(Yv, q.x);
      double x1 = lo_op(X, q.y), y1 = hi_op(Yv, q.y);
      double x2 = lo_op(X, q.z), y2 = hi_op(Yv, q.z);
      double x3 = lo_op(X, q.w), y3 = hi_op(Yv, q.w);
      for (int32_t t = 0; t < T; ++t)
      {
        const uint4 q2 = (t + 2 < T) ? tq[(t + 2) * n] : qn;
        const double u0 = lo_op(X, qn.x), v0 = hi_op(Yv, qn.x);
        const double u1 = lo_op(X, qn.y), v1 = hi_op(Yv, qn.y);
        const double u2 = lo_op(X, qn.z), v2 = hi_op(Yv, qn.z);
        const double u3 = lo_op(X, qn.w), v3 = hi_op(Yv, qn.w);
        acc[0] -= x0 * y0;
        acc[1] -= x1 * y1;
        acc[2] -= x2 * y2;
        acc[3] -= x3 * y3;
        x0 = u0;
        y0 = v0;
        x1 = u1;
        y1 = v1;
        x2 = u2;
        y2 = v2;
        x3 = u3;
        y3 = v3;
        qn = q2;
      }
    }

    // One streamed block.  `acc` carries unfinished sums into the next block.
    template<int KIND>
    __device__ __forceinline__ void blk_run(const uint8_t* blk, const double* X, const double* Yv, double* out,
                                            double* inv, double alpha, double (&acc)[4], int lane)
    {
      const int32_t nseg = *reinterpret_cast<const int32_t*>(blk);
      const uint8_t* p = blk + 16;
      int4 d = *reinterpret_cast<const int4*>(p);
      for (int32_t g = 0; g < nseg; ++g)
      {
        const uint8_t* pn = p + d.z;
        const int4 dn = (g + 1 < nseg) ? *reinterpret_cast<const int4*>(pn) : d;
        const int32_t T = d.x, n = d.y & 0xFF, flags = (d.y >> 8) & 0xFF, U = d.y >> 16;
        if (lane < n)
        {
          const uint32_t* items = reinterpret_cast<const uint32_t*>(p + 16) + lane;
          const uint4* tq = reinterpret_cast<const uint4*>(p + 16 + Pad16(4 * n * U)) + lane;
          if (U == 1)
          {
            const uint32_t it = items[0];
            if (flags & kSegFirst)
              acc[0] = init_value<KIND>(it, out);
            const double fin = (flags & kSegLast) ? fin_operand<KIND>(it, X, inv) : 1.0;
            acc[0] = seg_chain(tq, n, T, X, Yv, acc[0]);
            if (flags & kSegLast)
              finalize<KIND>(it, acc[0], fin, out, inv, alpha, flags);
          }
          else
          {
            uint32_t it[4];
            double fin[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
              it[u] = items[u * n];
              const bool real = it[u] != kNoItem;
              if (flags & kSegFirst)
                acc[u] = real ? init_value<KIND>(it[u], out) : 0.0;
              fin[u] = (real && (flags & kSegLast)) ? fin_operand<KIND>(it[u], X, inv) : 1.0;
            }
            seg_chain4(tq, n, T, X, Yv, acc);
            if (flags & kSegLast)
            {
#pragma unroll
              for (int u = 0; u < 4; ++u)
                if (it[u] != kNoItem)
                  finalize<KIND>(it[u], acc[u], fin[u], out, inv, alpha, flags);
            }
          }
        }
        if (flags & kSegLevelEnd)
          __syncwarp();
        p = pn;
        d = dn;
      }
    }
  }  // namespace stream
}  // namespace micmb
