// Request-serving runtime (tb_server_*): factor and solve requests over a set
// of registered sparsity patterns, run with continuous batching on one GPU.
//
// - A fixed number of slots (worker threads) take requests from one queue;
//   every matrix's handle runs on its own CUDA stream.  A slot that finishes takes the oldest
//   queued request that can run now, so requests that arrive while others are
//   on the GPU start as soon as a slot and memory are free, and the work of
//   different slots overlaps on the device.
// - A request can run when its matrix is not in use by another slot (a
//   factorization handle is not re-entrant) and the matrix's device
//   footprint fits under the HBM cap: resident factors of idle matrices are
//   evicted, least recently used first, to make room.
// - Factors stay resident between requests, so a solve-only request on a
//   resident matrix costs one refined solve; if the factor was evicted it is
//   recomputed from the matrix's last values first.
// - Every handle runs in the mixed-precision mode (FP32 factor, FP64
//   refinement to the request's tolerance) unless the server was created for
//   FP64.
#include "tensors_b200.h"
#include "common.hpp"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace
{

using Clock = std::chrono::steady_clock;

struct Matrix
{
    std::int32_t n = 0;
    std::vector<std::int64_t> outer;
    std::vector<std::int32_t> inner;
    std::vector<std::int32_t> perm;
    bool has_perm = false;
    std::vector<double> values;          // values of the last factorization (for refactoring after eviction)
    double reg = 0.0;
    tb_chol * h = nullptr;
    bool busy = false;
    bool factored = false;
    std::int64_t bytes = 0;              // device bytes reserved or held while resident
    std::int64_t estimate = 0;           // footprint: the caller's estimate, then the largest measured
    std::uint64_t last_use = 0;
};

struct Request
{
    std::int64_t id = 0;
    std::int64_t matrix = 0;
    bool factor = false;
    std::vector<double> values;
    double reg = 0.0;
    const double * B = nullptr;
    double * X = nullptr;
    std::int32_t nrhs = 1;
    double tol = 1e-10;
    int status = 1;                      // 1 = pending
    std::string error;
    std::int32_t iterations = 0;
    double relres = 0.0;
    Clock::time_point t_submit, t_start, t_end;
    bool done = false;
};

} // namespace

struct tb_server
{
    int device = 0;
    int precision = TB_PRECISION_MIXED;
    std::int64_t cap = 0;
    std::int64_t resident = 0;
    std::int64_t peak_resident = 0;
    std::uint64_t tick = 0;
    std::int64_t next_id = 0;
    bool stopping = false;
    std::vector<std::unique_ptr<Matrix>> matrices;
    std::deque<Request *> queue;
    std::map<std::int64_t, std::unique_ptr<Request>> requests;
    std::int64_t evictions = 0, refactors = 0;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::vector<std::thread> workers;

    ~tb_server()
    {
        {
            std::lock_guard<std::mutex> lk( m );
            stopping = true;
        }
        cv_work.notify_all();
        for( auto & w : workers ) { w.join(); }
        for( auto & mx : matrices ) { if( mx->h ) { tb_chol_destroy( mx->h ); } }
    }

    // Under the lock: make `need` bytes fit by evicting idle resident matrices
    // (least recently used first).  False if even then it does not fit.
    bool make_room( std::int64_t need, const Matrix * keep )
    {
        while( resident + need > cap )
        {
            Matrix * victim = nullptr;
            for( auto & mx : matrices )
            {
                if( mx.get() == keep || mx->busy || mx->h == nullptr ) { continue; }
                if( victim == nullptr || mx->last_use < victim->last_use ) { victim = mx.get(); }
            }
            if( victim == nullptr ) { return false; }
            tb_chol_destroy( victim->h );
            victim->h = nullptr;
            victim->factored = false;
            resident -= victim->bytes;
            victim->bytes = 0;
            ++evictions;
        }
        return true;
    }

    // Under the lock: the oldest queued request that can start now.
    Request * take()
    {
        for( auto it = queue.begin(); it != queue.end(); ++it )
        {
            Request * r = *it;
            Matrix * mx = matrices[static_cast<size_t>( r->matrix )].get();
            if( mx->busy ) { continue; }
            const std::int64_t need = mx->h ? 0 : mx->estimate;
            if( need > 0 && !make_room( need, mx ) ) { continue; }
            mx->busy = true;
            if( need > 0 ) { resident += need; mx->bytes = need; }   // reserved; corrected to the measured size afterwards
            peak_resident = std::max( peak_resident, resident );
            queue.erase( it );
            return r;
        }
        return nullptr;
    }

    void run( Request * r )
    {
        Matrix * mx = matrices[static_cast<size_t>( r->matrix )].get();
        r->t_start = Clock::now();
        int st = TB_OK;
        if( mx->h == nullptr )
        {
            st = tb_chol_create( &mx->h, mx->n, mx->outer.data(), mx->inner.data(),
                                 mx->has_perm ? mx->perm.data() : nullptr, 0 );
            if( st == TB_OK ) { st = tb_chol_set_precision( mx->h, precision ); }
            mx->factored = false;
        }
        if( st == TB_OK && r->factor )
        {
            mx->values = r->values;
            mx->reg = r->reg;
        }
        if( st == TB_OK && (r->factor || !mx->factored) )
        {
            if( mx->values.empty() ) { st = TB_ERR_NOT_FACTORIZED; }
            else
            {
                if( !r->factor ) { ++refactors; }
                st = tb_chol_numeric( mx->h, mx->values.data(), mx->reg );
                mx->factored = (st == TB_OK);
            }
        }
        if( st == TB_OK && r->B != nullptr )
        {
            st = tb_chol_set_refinement( mx->h, r->tol, 200 );
            if( st == TB_OK ) { st = tb_chol_solve( mx->h, 1.0, r->B, r->nrhs, 0.0, r->X, r->nrhs, r->nrhs ); }
            tb_chol_refinement_info( mx->h, &r->iterations, &r->relres );
        }
        if( st != TB_OK ) { r->error = tb_last_error(); }
        r->t_end = Clock::now();
        std::int64_t bytes = 0;
        if( mx->h ) { tb_chol_device_bytes( mx->h, &bytes ); }
        std::lock_guard<std::mutex> lk( m );
        resident += bytes - mx->bytes;
        mx->bytes = bytes;
        mx->estimate = std::max( mx->estimate, bytes );
        peak_resident = std::max( peak_resident, resident );
        mx->busy = false;
        mx->last_use = ++tick;
        r->status = st;
        r->done = true;
        cv_done.notify_all();
        cv_work.notify_all();
    }

    void worker()
    {
        tb_set_device( device );
        cudaSetDevice( device );
        for( ;; )
        {
            Request * r = nullptr;
            {
                std::unique_lock<std::mutex> lk( m );
                cv_work.wait( lk, [&] { return stopping || (r = take()) != nullptr; } );
                if( r == nullptr ) { break; }
            }
            run( r );
        }
    }
};

namespace
{

int sfail( int code, const std::string & msg )
{
    tb::set_last_error( msg );
    return code;
}

} // namespace

extern "C" {

int tb_server_create( tb_server ** out, int device, int64_t hbm_cap_bytes, int32_t slots, int32_t precision )
{
    if( out == nullptr || hbm_cap_bytes <= 0 || slots <= 0 || slots > 64 )
    {
        return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_create: cap > 0 and 1 <= slots <= 64 required" );
    }
    if( precision != TB_PRECISION_FP64 && precision != TB_PRECISION_MIXED )
    {
        return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_create: unknown precision" );
    }
    tb_server * s = new tb_server();
    s->device = device;
    s->cap = hbm_cap_bytes;
    s->precision = precision;
    for( int i = 0; i < slots; ++i ) { s->workers.emplace_back( [s] { s->worker(); } ); }
    *out = s;
    return TB_OK;
}

int tb_server_destroy( tb_server * s )
{
    delete s;
    return TB_OK;
}

int tb_server_add_matrix( tb_server * s, int32_t n, const int64_t * outer, const int32_t * inner, const int32_t * perm,
                          int64_t footprint_bytes, int64_t * matrix_id )
{
    if( s == nullptr || n <= 0 || outer == nullptr || inner == nullptr || matrix_id == nullptr || footprint_bytes <= 0 )
    {
        return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_add_matrix: invalid argument" );
    }
    auto mx = std::make_unique<Matrix>();
    mx->n = n;
    mx->outer.assign( outer, outer + n + 1 );
    mx->inner.assign( inner, inner + outer[n] );
    if( perm ) { mx->perm.assign( perm, perm + n ); mx->has_perm = true; }
    mx->estimate = footprint_bytes;
    std::lock_guard<std::mutex> lk( s->m );
    *matrix_id = static_cast<int64_t>( s->matrices.size() );
    s->matrices.push_back( std::move( mx ) );
    return TB_OK;
}

int tb_server_submit( tb_server * s, int64_t matrix_id, const double * values, double reg, const double * B, double * X,
                      int32_t nrhs, double tol, int64_t * request_id )
{
    if( s == nullptr || request_id == nullptr ) { return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_submit: null argument" ); }
    if( (B == nullptr) != (X == nullptr) || (B == nullptr && values == nullptr) )
    {
        return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_submit: a request factors (values), solves (B and X), or both" );
    }
    auto r = std::make_unique<Request>();
    {
        std::lock_guard<std::mutex> lk( s->m );
        if( matrix_id < 0 || matrix_id >= static_cast<int64_t>( s->matrices.size() ) )
        {
            return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_submit: unknown matrix" );
        }
        const Matrix * mx = s->matrices[static_cast<size_t>( matrix_id )].get();
        if( mx->estimate > s->cap ) { return sfail( TB_ERR_OUT_OF_MEMORY, "tb_server_submit: matrix footprint exceeds the HBM cap" ); }
        r->id = s->next_id++;
    }
    r->matrix = matrix_id;
    r->factor = values != nullptr;
    if( values )
    {
        std::lock_guard<std::mutex> lk( s->m );
        const Matrix * mx = s->matrices[static_cast<size_t>( matrix_id )].get();
        r->values.assign( values, values + mx->outer[static_cast<size_t>( mx->n )] );
    }
    r->reg = reg;
    r->B = B;
    r->X = X;
    r->nrhs = nrhs < 1 ? 1 : nrhs;
    r->tol = tol;
    r->t_submit = Clock::now();
    *request_id = r->id;
    {
        std::lock_guard<std::mutex> lk( s->m );
        s->queue.push_back( r.get() );
        s->requests[r->id] = std::move( r );
    }
    s->cv_work.notify_one();
    return TB_OK;
}

// Waits for a request: its status (TB_OK, a solve / factorization status),
// queue + run latency and run time (ms), refinement steps and residual.
int tb_server_wait( tb_server * s, int64_t request_id, int32_t * status, double * latency_ms, double * run_ms,
                    int32_t * iterations, double * relres )
{
    if( s == nullptr ) { return sfail( TB_ERR_INVALID_ARGUMENT, "null server" ); }
    std::unique_lock<std::mutex> lk( s->m );
    auto it = s->requests.find( request_id );
    if( it == s->requests.end() ) { return sfail( TB_ERR_INVALID_ARGUMENT, "tb_server_wait: unknown request" ); }
    Request * r = it->second.get();
    s->cv_done.wait( lk, [&] { return r->done; } );
    if( status ) { *status = r->status; }
    if( latency_ms ) { *latency_ms = std::chrono::duration<double, std::milli>( r->t_end - r->t_submit ).count(); }
    if( run_ms ) { *run_ms = std::chrono::duration<double, std::milli>( r->t_end - r->t_start ).count(); }
    if( iterations ) { *iterations = r->iterations; }
    if( relres ) { *relres = r->relres; }
    if( r->status != TB_OK ) { tb::set_last_error( r->error ); }
    const int st = r->status;
    s->requests.erase( it );
    return st == TB_OK ? TB_OK : st;
}

// Resident bytes now, the peak so far, evictions and refactorizations after eviction.
int tb_server_stats( tb_server * s, int64_t * resident, int64_t * peak, int64_t * evictions, int64_t * refactors )
{
    if( s == nullptr ) { return sfail( TB_ERR_INVALID_ARGUMENT, "null server" ); }
    std::lock_guard<std::mutex> lk( s->m );
    if( resident ) { *resident = s->resident; }
    if( peak ) { *peak = s->peak_resident; }
    if( evictions ) { *evictions = s->evictions; }
    if( refactors ) { *refactors = s->refactors; }
    return TB_OK;
}

} // extern "C"
