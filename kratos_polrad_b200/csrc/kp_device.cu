// Device layer of the C ABI: thin, checked wrappers over the CUDA runtime.
// Replaces device::base_t's function objects and stream/event virtuals
// (src/device/device.h:37-186) and cuda_t (src/device/cuda/cuda.cpp).
#include "kp_common.cuh"

namespace kp
{
static thread_local std::string g_last_error;
void set_last_error( const std::string & msg ) { g_last_error = msg; }
void clear_last_error(  ) { g_last_error.clear(  ); }
}

using kp::guarded;
using kp::require;

extern "C" {

const char * kp_last_error( void ) { return kp::g_last_error.c_str(  ); }
int kp_abi_version( void ) { return KP_ABI_VERSION; }

int kp_device_init( int idx_device )
{
    return guarded( "kp_device_init", [ & ]
    {
        int n = 0;
        KP_CUDA( cudaGetDeviceCount( & n ) );
        require( idx_device >= 0 && idx_device < n, "device index out of range" );
        KP_CUDA( cudaSetDevice( idx_device ) );
        KP_CUDA( cudaFree( nullptr ) );          // create the context now
    } );
}

int kp_device_count( int * n )
{
    return guarded( "kp_device_count", [ & ]
    {
        require( n != nullptr, "n is null" );
        KP_CUDA( cudaGetDeviceCount( n ) );
    } );
}

int kp_malloc( void ** p, size_t bytes )
{
    return guarded( "kp_malloc", [ & ]
    {
        require( p != nullptr, "p is null" );
        * p = nullptr;
        if( bytes == 0 ) return;
        const cudaError_t e = cudaMalloc( p, bytes );
        if( e == cudaErrorMemoryAllocation )
        {
            cudaGetLastError(  );
            throw kp::error_t( KP_ERR_ALLOC, "device allocation refused" );
        }
        KP_CUDA( e );
    } );
}

int kp_malloc_host( void ** p, size_t bytes )
{
    return guarded( "kp_malloc_host", [ & ]
    {
        require( p != nullptr, "p is null" );
        * p = nullptr;
        if( bytes == 0 ) return;
        KP_CUDA( cudaMallocHost( p, bytes ) );
    } );
}

int kp_free( void * p )
{
    return guarded( "kp_free", [ & ] { if( p ) KP_CUDA( cudaFree( p ) ); } );
}

int kp_free_host( void * p )
{
    return guarded( "kp_free_host", [ & ] { if( p ) KP_CUDA( cudaFreeHost( p ) ); } );
}

int kp_memset_async( void * p, int value, size_t bytes, void * stream )
{
    return guarded( "kp_memset_async", [ & ]
    {
        KP_CUDA( cudaMemsetAsync( p, value, bytes, ( cudaStream_t ) stream ) );
    } );
}

int kp_memcpy( void * dst, const void * src, size_t bytes )
{
    return guarded( "kp_memcpy", [ & ]
    {
        KP_CUDA( cudaMemcpy( dst, src, bytes, cudaMemcpyDefault ) );
    } );
}

int kp_memcpy_async( void * dst, const void * src, size_t bytes, void * stream )
{
    return guarded( "kp_memcpy_async", [ & ]
    {
        KP_CUDA( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyDefault,
                                  ( cudaStream_t ) stream ) );
    } );
}

int kp_stream_create( void ** stream )
{
    return guarded( "kp_stream_create", [ & ]
    {
        require( stream != nullptr, "stream is null" );
        cudaStream_t s;
        KP_CUDA( cudaStreamCreateWithFlags( & s, cudaStreamNonBlocking ) );
        * stream = s;
    } );
}

int kp_stream_destroy( void * stream )
{
    return guarded( "kp_stream_destroy", [ & ]
    {
        if( stream ) KP_CUDA( cudaStreamDestroy( ( cudaStream_t ) stream ) );
    } );
}

int kp_stream_sync( void * stream )
{
    return guarded( "kp_stream_sync", [ & ]
    {
        KP_CUDA( cudaStreamSynchronize( ( cudaStream_t ) stream ) );
    } );
}

int kp_event_create( void ** event )
{
    return guarded( "kp_event_create", [ & ]
    {
        require( event != nullptr, "event is null" );
        cudaEvent_t e;
        KP_CUDA( cudaEventCreate( & e ) );
        * event = e;
    } );
}

int kp_event_destroy( void * event )
{
    return guarded( "kp_event_destroy", [ & ]
    {
        if( event ) KP_CUDA( cudaEventDestroy( ( cudaEvent_t ) event ) );
    } );
}

int kp_event_record( void * event, void * stream )
{
    return guarded( "kp_event_record", [ & ]
    {
        KP_CUDA( cudaEventRecord( ( cudaEvent_t ) event, ( cudaStream_t ) stream ) );
    } );
}

int kp_event_wait( void * stream, void * event )
{
    return guarded( "kp_event_wait", [ & ]
    {
        KP_CUDA( cudaStreamWaitEvent( ( cudaStream_t ) stream,
                                      ( cudaEvent_t ) event, 0 ) );
    } );
}

int kp_event_sync( void * event )
{
    return guarded( "kp_event_sync", [ & ]
    {
        KP_CUDA( cudaEventSynchronize( ( cudaEvent_t ) event ) );
    } );
}

int kp_event_elapsed( float * ms, void * start, void * stop )
{
    return guarded( "kp_event_elapsed", [ & ]
    {
        require( ms != nullptr, "ms is null" );
        KP_CUDA( cudaEventElapsedTime( ms, ( cudaEvent_t ) start,
                                       ( cudaEvent_t ) stop ) );
    } );
}

int kp_launch_host( void * stream, void ( * fn )( void * ), void * arg )
{
    return guarded( "kp_launch_host", [ & ]
    {
        require( fn != nullptr, "fn is null" );
        KP_CUDA( cudaLaunchHostFunc( ( cudaStream_t ) stream, fn, arg ) );
    } );
}

}   // extern "C"
