/* Host compatibility shim for compiling the reference's CUDA-in-.cpp
 * traversal code with g++ (test infrastructure only; never shipped).
 *
 * The reference compiles every .cpp as CUDA (`nvcc -x cu`, Makefile:22-36).
 * Its packet traversal (photon.h, proxy.h, particle_base.h, geometry.h,
 * dat_3d.h) only needs the CUDA function-space qualifiers, `dim3`, the
 * thread-index builtins and `atomicAdd` to be defined; this header supplies
 * host stand-ins so that the very same source runs one packet at a time on
 * the CPU.  Deposits made through `atomicAdd` are forwarded to a hook that
 * the harness defines, which records them both as the reference's float sum
 * and as an order-independent int64 fixed-point sum.
 */
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>

#define __host__
#define __device__
#define __global__
#define __constant__
#define __shared__
#define __forceinline__ inline

struct dim3
{
    unsigned x, y, z;
    dim3( unsigned a = 1, unsigned b = 1, unsigned c = 1 )
        : x( a ), y( b ), z( c ) {}
};
struct kp_ref_tid_t { unsigned x = 0, y = 0, z = 0; };
static kp_ref_tid_t threadIdx, blockIdx, blockDim, gridDim;

/* Deposit hook: defined by ref_harness.cpp. */
void kp_ref_deposit( float  * p, float  v );
void kp_ref_deposit( double * p, double v );
inline float  atomicAdd( float  * p, float  v )
{ float  o = * p; kp_ref_deposit( p, v ); return o; }
inline double atomicAdd( double * p, double v )
{ double o = * p; kp_ref_deposit( p, v ); return o; }
template< class T > inline T atomicAdd( T * p, T v )
{ T o = * p; * p = o + v; return o; }
template< class T > inline T atomicCAS( T * p, T c, T v )
{ T o = * p; if( o == c ) * p = v; return o; }

#define __dyn_shared__( T, N ) T * N = nullptr

namespace device
{
struct kp_ref_stream_opaque;
struct kp_ref_event_opaque;
using stream_t = kp_ref_stream_opaque *;
using event_t  = kp_ref_event_opaque  *;
}
