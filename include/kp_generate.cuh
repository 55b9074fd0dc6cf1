// kratos_polrad_b200 — user packet generators, for CUDA translation units.
//
// The reference launches the user's generator functor once per packet of a
// cycle (generate::ker_gen over n_par threads, modules/particle/evolve/
// generate_par.h:10-15, 51-62); the functor writes each packet's position,
// direction, cell, block and weight into the pool.  Here the user's functor
//
//     struct my_gen_t
//     {
//         __device__ void operator()( kp_packet_init_t & pk, long long pid ) const;
//     };
//
// is launched the same way over a table of kp_packet_init_t, which
// kp_transport_cfg_t::packets then hands to the walk: it sets pk.x, pk.d
// (unit), pk.w, optionally pk.stokes and pk.peel_I, and pk.ib (or -1 to let
// the walk locate the position).  `pid` is the packet's global id, the key
// of its RNG stream in the walk.  Compile with nvcc (sm_100a); include
// kp_module.hpp to enroll the generator in the radiation module.
#ifndef KP_GENERATE_CUH
#define KP_GENERATE_CUH

#include "kp_transport.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace kp::generate
{

template< class gen_T >
__global__ void ker_gen( const gen_T gen, kp_packet_init_t * table, long long n, long long pid0 )
{
    const long long i = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    if( i < n )
        gen( table[ i ], pid0 + i );
}

// Fills table[0 .. n) (device memory) for packets pid0 .. pid0 + n - 1 on
// `stream`, n_th threads per block (the reference's [particle] n_th).
template< class gen_T >
void launch( const gen_T & gen, kp_packet_init_t * table, long long n, long long pid0,
             void * stream, int n_th = 64 )
{
    if( n <= 0 )
        return;
    if( n_th < 32 || n_th > 1024 || n_th % 32 )
        throw std::runtime_error( "kratos_polrad_b200: generator threads per block must be a "
                                  "multiple of 32 in 32..1024" );
    const long long n_bl = ( n + n_th - 1 ) / n_th;
    if( n_bl > 0x7fffffffLL )
        throw std::runtime_error( "kratos_polrad_b200: too many packets for one generator launch" );
    ker_gen<<< ( unsigned ) n_bl, ( unsigned ) n_th, 0, ( cudaStream_t ) stream >>>( gen, table, n,
                                                                                    pid0 );
    const cudaError_t e = cudaGetLastError(  );
    if( e != cudaSuccess )
        throw std::runtime_error( std::string( "kratos_polrad_b200: generator launch: " )
                                  + cudaGetErrorString( e ) );
}

// A device functor as the radiation module's generator hook
// (kp::particle::radiation::base_t::enroll).
template< class gen_T >
struct on_device_t
{
    gen_T gen;
    int   n_th;
    void operator()( kp_packet_init_t * table, long long n, long long pid0, void * s ) const
    {
        launch( gen, table, n, pid0, s, n_th );
    }
};

template< class gen_T >
on_device_t< gen_T > on_device( const gen_T & gen, int n_th = 64 )
{
    return on_device_t< gen_T > { gen, n_th };
}

}   // namespace kp::generate

#endif
