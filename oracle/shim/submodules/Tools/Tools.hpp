#pragma once
// Project-written stand-in for the utility library that the reference
// headers include as "submodules/Tools/Tools.hpp".  That submodule is an
// empty directory in the reference checkout (its .gitmodules entry pins no
// commit), so the names the Cholesky path uses are written here from their
// call-site meaning only: containers' allocation helpers, buffer kernels,
// thread-loop drivers, scalar traits, enums and logging.  It is test
// infrastructure: it lets oracle/ compile the reference's own headers into a
// CPU checker and baseline (oracle/_ref); nothing in the product includes it.
//
// Thread loops run on std::thread; every parallel loop here is a plain
// fork-join over contiguous chunks, which is all the call sites need.

#include <algorithm>
#include <any>
#include <atomic>
#include <cassert>
#include <chrono>
#include <cmath>
#include <complex>
#include <concepts>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <typeinfo>
#include <utility>
#include <vector>

#define TOOLS_FORCE_INLINE inline
#define TOOLS_RESTRICT __restrict
#define TOOLS_DEBUG_ASSERT(c, msg)
#define TOOLS_DEBUG_PRINT(msg)
#define TOOLS_MAKE_FP_FAST()
#define TOOLS_MAKE_FP_STRICT()

namespace Tools
{
    using Size_T = std::size_t;
    using Int8   = std::int8_t;
    using Int16  = std::int16_t;
    using Int32  = std::int32_t;
    using Int64  = std::int64_t;
    using UInt8  = std::uint8_t;
    using UInt32 = std::uint32_t;
    using UInt64 = std::uint64_t;
    using Real32 = float;
    using Real64 = double;

    constexpr Size_T VarSize          = 0;
    constexpr Size_T DefaultAlignment = 64;
    constexpr Size_T ObjectAlignment  = 64;

    template<typename T> using cptr = const T * TOOLS_RESTRICT;
    template<typename T> using mptr = T * TOOLS_RESTRICT;
    template<typename T> using cref = const T &;
    template<typename T> using mref = T &;

    template<typename T> concept IntQ       = std::integral<T>;
    template<typename T> concept SignedIntQ = std::integral<T> && std::is_signed_v<T>;
    template<typename A, typename B> constexpr bool SameQ = std::is_same_v<A,B>;
    template<typename T> constexpr bool ArithmeticQ = std::is_arithmetic_v<T>;

    enum Parallel_T : bool { Sequential = false, Parallel = true };

    enum class Op     : int { Id = 0, Trans = 1, ConjTrans = 2, Conj = 3, Re = 4, ReTrans = 5, Im = 6, ImTrans = 7 };
    enum class Layout : int { RowMajor = 0, ColMajor = 1 };
    enum class UpLo   : int { Upper = 0, Lower = 1 };
    enum class Side   : int { Left = 0, Right = 1 };
    enum class Diag   : int { NonUnit = 0, Unit = 1 };

    constexpr UpLo Transpose( UpLo u ) { return u == UpLo::Upper ? UpLo::Lower : UpLo::Upper; }
    constexpr Op   Transpose( Op o )   { return o == Op::Id ? Op::Trans : Op::Id; }

    constexpr Size_T CacheLineWidth = 64;

    // For static_assert(false-like) in discarded constexpr branches.
    template<typename...> constexpr bool DependentFalse = false;

    // max(x, 0)
    template<typename T> constexpr T Ramp( const T x ) { return x > T(0) ? x : T(0); }

    // ---------------------------------------------------------------- scalars
    namespace Scalar
    {
        template<typename T> struct RealOf { using type = T; };
        template<typename T> struct RealOf<std::complex<T>> { using type = T; };
        template<typename T> using Real = typename RealOf<T>::type;

        template<typename T> constexpr bool ComplexQ = !std::is_same_v<T, Real<T>>;
        template<typename T> constexpr bool RealQ    = std::is_floating_point_v<T>;
        template<typename T> constexpr bool FloatQ   = std::is_floating_point_v<Real<T>>;

        template<typename T> constexpr T Zero = T(0);
        template<typename T> constexpr T One  = T(1);
        template<typename T> constexpr T Two  = T(2);
        template<typename T> constexpr T Half = T(0.5);

        template<typename T> constexpr T Max = std::numeric_limits<T>::max();
        template<typename T> constexpr T Min = std::numeric_limits<T>::lowest();
        template<typename T> constexpr T Infty = std::numeric_limits<T>::infinity();
        template<typename T> constexpr T eps = std::numeric_limits<T>::epsilon();

        // How a coefficient in a linear combination is to be treated.
        enum class Flag : int { Zero = 0, Plus = 1, Minus = -1, Generic = 2 };

        // An entry under an operation (MatrixCSR's transpose and real/imaginary parts).
        template<::Tools::Op op, typename T> constexpr T Op( const T & x )
        {
            if constexpr ( op == ::Tools::Op::Conj || op == ::Tools::Op::ConjTrans )
            {
                if constexpr ( ComplexQ<T> ) { return std::conj(x); } else { return x; }
            }
            else if constexpr ( op == ::Tools::Op::Re || op == ::Tools::Op::ReTrans )
            {
                if constexpr ( ComplexQ<T> ) { return T(std::real(x)); } else { return x; }
            }
            else if constexpr ( op == ::Tools::Op::Im || op == ::Tools::Op::ImTrans )
            {
                if constexpr ( ComplexQ<T> ) { return T(std::imag(x)); } else { return T(0); }
            }
            else { return x; }
        }
    }
    using Complex32 = std::complex<float>;
    using Complex64 = std::complex<double>;

    template<typename T> inline T Max( const T a, const T b ) { return a < b ? b : a; }
    template<typename T> inline T Min( const T a, const T b ) { return a < b ? a : b; }
    template<typename T> inline auto Abs( const T x ) { return std::abs(x); }
    template<typename T> inline T Sqrt( const T x ) { return std::sqrt(x); }
    template<typename T> inline T Inv( const T x ) { return T(1) / x; }
    template<typename T> inline T Frac( const T a, const T b ) { return a / b; }
    template<typename T> inline T Conj( const T x )
    {
        if constexpr ( Scalar::ComplexQ<T> ) { return std::conj(x); } else { return x; }
    }
    template<typename T> inline auto Re( const T x )
    {
        if constexpr ( Scalar::ComplexQ<T> ) { return std::real(x); } else { return x; }
    }
    template<typename T> inline auto Im( const T x )
    {
        if constexpr ( Scalar::ComplexQ<T> ) { return std::imag(x); } else { return T(0); }
    }
    template<typename T> inline bool NaNQ( const T x ) { return std::isnan(Re(x)); }

    template<typename T, typename S> inline T int_cast( const S x ) { return static_cast<T>(x); }
    template<typename S> inline Size_T ToSize_T( const S x ) { return static_cast<Size_T>(x); }

    // ------------------------------------------------------------------ names
    template<typename T> inline std::string TypeNameOf()
    {
        if constexpr ( std::is_same_v<T,double> )              { return "Real64"; }
        else if constexpr ( std::is_same_v<T,float> )          { return "Real32"; }
        else if constexpr ( std::is_same_v<T,std::int32_t> )   { return "Int32"; }
        else if constexpr ( std::is_same_v<T,std::int64_t> )   { return "Int64"; }
        else if constexpr ( std::is_same_v<T,long long> )      { return "Int64"; }
        else if constexpr ( std::is_same_v<T,bool> )           { return "Bool"; }
        else { return typeid(T).name(); }
    }
    template<typename T> inline const std::string TypeName = TypeNameOf<T>();

    inline std::string ToString( const std::string & s ) { return s; }
    inline std::string ToString( const char * s ) { return std::string(s); }
    inline std::string ToString( const bool b ) { return b ? "true" : "false"; }
    inline std::string ToString( const Parallel_T p ) { return p == Parallel ? "Parallel" : "Sequential"; }
    inline std::string ToString( const Op o ) { return std::to_string(static_cast<int>(o)); }
    inline std::string ToString( const Layout o ) { return std::to_string(static_cast<int>(o)); }
    inline std::string ToString( const UpLo o ) { return std::to_string(static_cast<int>(o)); }
    inline std::string ToString( const Side o ) { return std::to_string(static_cast<int>(o)); }
    inline std::string ToString( const Diag o ) { return std::to_string(static_cast<int>(o)); }
    template<typename T>
    inline std::enable_if_t<std::is_arithmetic_v<T>,std::string> ToString( const T x )
    {
        std::ostringstream s; s << x; return s.str();
    }
    template<typename T>
    inline std::enable_if_t<std::is_enum_v<T>,std::string> ToString( const T x )
    {
        return std::to_string(static_cast<long long>(x));
    }

    // ---------------------------------------------------------------- logging
    inline bool & LogQuiet() { static bool q = false; return q; }
    inline void print( const std::string & s ) { if( !LogQuiet() ) { std::cout << s << std::endl; } }
    inline void eprint( const std::string & s ) { if( !LogQuiet() ) { std::cerr << "ERROR: " << s << std::endl; } }
    inline void wprint( const std::string & s ) { if( !LogQuiet() ) { std::cerr << "WARNING: " << s << std::endl; } }
    inline void logprint( const std::string & ) {}
    template<typename T> inline void logvalprint( const std::string &, const T & ) {}
    template<typename T> inline void valprint( const std::string &, const T & ) {}
    inline void tic( const std::string & ) {}
    inline void toc( const std::string & ) {}

    namespace Format { namespace Matrix { constexpr int TSV = 0; } }

    struct OutString
    {
        template<typename... Args> static std::string FromMatrix( Args&&... ) { return std::string(); }
        template<typename... Args> static std::string FromVector( Args&&... ) { return std::string(); }
        template<typename... Args> static std::string FromArray( Args&&... ) { return std::string(); }
        template<int fmt, typename... Args> static std::string FromMatrix( Args&&... ) { return std::string(); }
    };

    template<typename T> inline void assert_positive( const T ) {}

#define TOOLS_DUMP(x)
#define TOOLS_LOGDUMP(x)
#define TOOLS_DDUMP(x)
#define TOOLS_PDUMP(x)
#define TOOLS_PTIMER(timer, tag)
#define TOOLS_PTIC(tag)
#define TOOLS_PTOC(tag)

    struct Profiler { static void Clear() {} };

    using Clock = std::chrono::steady_clock;
    using Time  = std::chrono::time_point<Clock>;
    inline double Duration( const Time & a, const Time & b )
    {
        return std::chrono::duration<double>(b - a).count();
    }

    // ------------------------------------------------------------- allocation
    template<typename P>
    inline void safe_alloc( P & a, const Size_T n, const Size_T alignment = DefaultAlignment )
    {
        using T = std::remove_cv_t<std::remove_reference_t<decltype(*a)>>;
        if( a != nullptr ) { std::free(a); a = nullptr; }
        const Size_T bytes = ((Max<Size_T>(n,1) * sizeof(T) + alignment - 1) / alignment) * alignment;
        a = static_cast<T*>( std::aligned_alloc( alignment, bytes ) );
    }
    template<typename P>
    inline void safe_free( P & a )
    {
        if( a != nullptr ) { std::free(a); a = nullptr; }
    }

    // ------------------------------------------------------------ thread loops
    template<typename I>
    inline I JobPointer( const I n, const I thread_count, const I thread )
    {
        // Even split of [0,n) into thread_count contiguous chunks.
        return static_cast<I>( (static_cast<long long>(n) * thread) / Max<I>(thread_count, I(1)) );
    }

    template<typename Int_>
    class JobPointers
    {
    public:
        using Int = Int_;
    private:
        std::vector<Int> ptr { Int(0), Int(0) };
    public:
        JobPointers() = default;

        template<typename I0, typename I1>
        JobPointers( const I0 job_count, const I1 thread_count )
        {
            const Int t = Max<Int>( Int(1), static_cast<Int>(thread_count) );
            ptr.assign( static_cast<Size_T>(t) + 1, Int(0) );
            for( Int k = 0; k <= t; ++k )
            {
                ptr[static_cast<Size_T>(k)] = JobPointer<Int>( static_cast<Int>(job_count), t, k );
            }
        }

        // Split [0,job_count) by a cumulative cost array (costs[0..job_count]).
        template<typename I0, typename C, typename I1>
        JobPointers( const I0 job_count, const C * costs, const I1 thread_count, const bool = true )
        {
            const Int m = static_cast<Int>(job_count);
            const Int t = Max<Int>( Int(1), static_cast<Int>(thread_count) );
            ptr.assign( static_cast<Size_T>(t) + 1, Int(0) );
            ptr[static_cast<Size_T>(t)] = m;
            if( m <= 0 ) { return; }
            const double c0 = static_cast<double>(costs[0]);
            const double total = static_cast<double>(costs[m]) - c0;
            for( Int k = 1; k < t; ++k )
            {
                const double target = c0 + total * static_cast<double>(k) / static_cast<double>(t);
                const C * pos = std::lower_bound( costs, costs + m + 1, static_cast<C>(target) );
                Int j = static_cast<Int>( pos - costs );
                j = Min<Int>( Max<Int>( j, ptr[static_cast<Size_T>(k-1)] ), m );
                ptr[static_cast<Size_T>(k)] = j;
            }
        }

        Int ThreadCount() const { return static_cast<Int>(ptr.size()) - 1; }
        Int operator[]( const Int k ) const { return ptr[static_cast<Size_T>(k)]; }
        const Int * data() const { return ptr.data(); }
        Int Size() const { return static_cast<Int>(ptr.size()); }
    };

    template<typename Int, Parallel_T parQ>
    inline Int TruncateThreadCount( const Int t )
    {
        return parQ == Parallel ? Max<Int>( Int(1), t ) : Int(1);
    }

    // Runs f(thread) for thread in [0,thread_count) on std::threads.
    template<typename F, typename I>
    inline void ParallelDo( F && f, const I thread_count )
    {
        const long long t = thread_count;
        if( t <= 1 ) { if( t == 1 ) { f( I(0) ); } return; }
        std::vector<std::thread> pool;
        pool.reserve( static_cast<Size_T>(t) );
        for( long long k = 0; k < t; ++k ) { pool.emplace_back( [&f,k](){ f( static_cast<I>(k) ); } ); }
        for( auto & th : pool ) { th.join(); }
    }

    // Runs f(i) for i in [0,n).
    template<Parallel_T parQ = Sequential, typename F, typename I, typename J>
    inline void Do( F && f, const I n, const J thread_count )
    {
        if( (parQ == Sequential) || (thread_count <= 1) || (n <= 1) )
        {
            for( I i = 0; i < n; ++i ) { f(i); }
            return;
        }
        const I t = static_cast<I>( Min<long long>( static_cast<long long>(thread_count), static_cast<long long>(n) ) );
        ParallelDo(
            [&]( const I thread )
            {
                const I b = JobPointer<I>( n, t, thread );
                const I e = JobPointer<I>( n, t, thread + 1 );
                for( I i = b; i < e; ++i ) { f(i); }
            },
            t
        );
    }

    // Runs f(i) for i in [0,n) over the chunks given by job pointers.
    template<Parallel_T parQ = Sequential, typename F, typename I>
    inline void Do( F && f, const JobPointers<I> & job_ptr )
    {
        const I t = job_ptr.ThreadCount();
        if( (parQ == Sequential) || (t <= 1) )
        {
            for( I i = job_ptr[0]; i < job_ptr[t]; ++i ) { f(i); }
            return;
        }
        ParallelDo(
            [&]( const I thread )
            {
                for( I i = job_ptr[thread]; i < job_ptr[thread+1]; ++i ) { f(i); }
            },
            t
        );
    }

    enum class Schedule_T : int { Static = 0, Dynamic = 1 };
    constexpr Schedule_T Static  = Schedule_T::Static;
    constexpr Schedule_T Dynamic = Schedule_T::Dynamic;

    // Runs f(thread, k) for k in [range.first, range.second) on thread_count
    // workers; with Dynamic, the workers take the next k from a shared counter.
    template<Parallel_T parQ, Schedule_T sched, typename F>
    inline void Do( F && f, const std::pair<Size_T,Size_T> range, const Size_T thread_count )
    {
        const Size_T b = range.first;
        const Size_T e = range.second;
        if( e <= b ) { return; }
        if( (parQ == Sequential) || (thread_count <= 1) )
        {
            for( Size_T k = b; k < e; ++k ) { f( Size_T(0), k ); }
            return;
        }
        std::atomic<Size_T> next { b };
        ParallelDo(
            [&]( const Size_T thread )
            {
                if constexpr ( sched == Schedule_T::Dynamic )
                {
                    for( Size_T k = next.fetch_add(1); k < e; k = next.fetch_add(1) ) { f( thread, k ); }
                }
                else
                {
                    const Size_T kb = b + JobPointer<Size_T>( e - b, thread_count, thread );
                    const Size_T ke = b + JobPointer<Size_T>( e - b, thread_count, thread + 1 );
                    for( Size_T k = kb; k < ke; ++k ) { f( thread, k ); }
                }
            },
            thread_count
        );
    }

    template<Parallel_T parQ = Sequential, typename F, typename R, typename T, typename I, typename J>
    inline T DoReduce( F && f, R && reduce, const T init, const I n, const J thread_count )
    {
        T result = init;
        if( (parQ == Sequential) || (thread_count <= 1) || (n <= 1) )
        {
            for( I i = 0; i < n; ++i ) { reduce( f(i), result ); }
            return result;
        }
        const I t = static_cast<I>( Min<long long>( static_cast<long long>(thread_count), static_cast<long long>(n) ) );
        std::vector<T> partial( static_cast<Size_T>(t), init );
        ParallelDo(
            [&]( const I thread )
            {
                const I b = JobPointer<I>( n, t, thread );
                const I e = JobPointer<I>( n, t, thread + 1 );
                T r = init;
                for( I i = b; i < e; ++i ) { reduce( f(i), r ); }
                partial[static_cast<Size_T>(thread)] = r;
            },
            t
        );
        for( const T & v : partial ) { reduce( v, result ); }
        return result;
    }

    template<typename F, typename R, typename T, typename I>
    inline T ParallelDoReduce( F && f, R && reduce, const T init, const I thread_count )
    {
        const I t = Max<I>( I(1), thread_count );
        std::vector<T> partial( static_cast<Size_T>(t), init );
        ParallelDo( [&]( const I thread ) { partial[static_cast<Size_T>(thread)] = f(thread); }, t );
        T result = init;
        for( const T & v : partial ) { reduce( v, result ); }
        return result;
    }

    // --------------------------------------------------------- buffer kernels
    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename S, typename T, typename I = Size_T>
    inline void copy_buffer( const S * from, T * to, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i ) { to[i] = static_cast<T>(from[i]); }
    }

    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename S, typename T, typename I = Size_T>
    inline void move_buffer( S * from, T * to, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i ) { to[i] = std::move(from[i]); }
    }

    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename T, typename S, typename I = Size_T>
    inline void fill_buffer( T * a, const S init, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i ) { a[i] = static_cast<T>(init); }
    }

    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename T, typename I = Size_T>
    inline void zerofy_buffer( T * a, const I n = static_cast<I>(N), const Size_T thread_count = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        if( (parQ == Parallel) && (thread_count > 1) )
        {
            Do<Parallel>( [=]( const Size_T i ) { a[i] = T(0); }, m, thread_count );
        }
        else
        {
            std::fill( a, a + m, T(0) );
        }
    }

    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename T, typename I = Size_T>
    inline void iota_buffer( T * a, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i ) { a[i] = static_cast<T>(i); }
    }

    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename A, typename T, typename I = Size_T>
    inline void scale_buffer( const A alpha, T * a, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i ) { a[i] = static_cast<T>(alpha) * a[i]; }
    }

    // y += x
    template<Size_T N = VarSize, Parallel_T parQ = Sequential, typename S, typename T, typename I = Size_T>
    inline void add_to_buffer( const S * x, T * y, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i ) { y[i] += static_cast<T>(x[i]); }
    }

    template<Scalar::Flag f, typename A, typename X>
    inline auto flagged_times( const A alpha, const X x )
    {
        if constexpr ( f == Scalar::Flag::Zero )  { return X(0); }
        else if constexpr ( f == Scalar::Flag::Plus )  { return x; }
        else if constexpr ( f == Scalar::Flag::Minus ) { return -x; }
        else { return alpha * x; }
    }

    template<Op op, typename X> inline X opval( const X x )
    {
        if constexpr ( op == Op::Conj || op == Op::ConjTrans ) { return Conj(x); } else { return x; }
    }

    // y = alpha * op(x) + beta * op(y); a Zero flag means the term is absent
    // (the old content of y is never read when beta's flag is Zero).
    template<
        Scalar::Flag a_flag, Scalar::Flag b_flag,
        Size_T N = VarSize, Parallel_T parQ = Sequential, Op opx = Op::Id, Op opy = Op::Id,
        typename A, typename S, typename B, typename T, typename I = Size_T
    >
    inline void combine_buffers(
        const A alpha, const S * x, const B beta, T * y, const I n = static_cast<I>(N), const Size_T = 1
    )
    {
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        for( Size_T i = 0; i < m; ++i )
        {
            T r = T(0);
            if constexpr ( a_flag != Scalar::Flag::Zero )
            {
                r += static_cast<T>( flagged_times<a_flag>( alpha, opval<opx>( static_cast<T>(x[i]) ) ) );
            }
            if constexpr ( b_flag != Scalar::Flag::Zero )
            {
                r += static_cast<T>( flagged_times<b_flag>( beta, opval<opy>( y[i] ) ) );
            }
            y[i] = r;
        }
    }

    template<
        Scalar::Flag a_flag, Scalar::Flag b_flag,
        Size_T M = VarSize, Size_T N = VarSize, Parallel_T parQ = Sequential, Op opx = Op::Id, Op opy = Op::Id,
        typename A, typename S, typename B, typename T, typename I, typename J, typename K, typename L
    >
    inline void combine_matrices(
        const A alpha, const S * X, const I ldX, const B beta, T * Y, const J ldY,
        const K m, const L n, const Size_T thread_count = 1
    )
    {
        Do<parQ>(
            [=]( const K i )
            {
                combine_buffers<a_flag,b_flag,N,Sequential,opx,opy>(
                    alpha, &X[static_cast<Size_T>(ldX) * static_cast<Size_T>(i)],
                    beta,  &Y[static_cast<Size_T>(ldY) * static_cast<Size_T>(i)], n
                );
            },
            m, thread_count
        );
    }

    template<Size_T M = VarSize, Size_T N = VarSize, Parallel_T parQ = Sequential,
        typename S, typename T, typename I, typename J, typename K, typename L>
    inline void copy_matrix( const S * X, const I ldX, T * Y, const J ldY, const K m, const L n, const Size_T thread_count = 1 )
    {
        Do<parQ>(
            [=]( const K i )
            {
                copy_buffer( &X[static_cast<Size_T>(ldX) * static_cast<Size_T>(i)],
                             &Y[static_cast<Size_T>(ldY) * static_cast<Size_T>(i)], n );
            },
            m, thread_count
        );
    }

    template<typename T, typename I>
    inline std::pair<T,T> minmax_buffer( const T * a, const I n, const Size_T = 1 )
    {
        if( n <= 0 ) { return { T(0), T(0) }; }
        auto r = std::minmax_element( a, a + n );
        return { *r.first, *r.second };
    }

    template<typename T, typename I>
    inline Scalar::Real<T> norm_max( const T * a, const I n, const Size_T = 1 )
    {
        Scalar::Real<T> r = 0;
        for( I i = 0; i < n; ++i ) { r = Max( r, static_cast<Scalar::Real<T>>(std::abs(a[i])) ); }
        return r;
    }

    // sum_i opx(x[i]) * opy(y[i])
    template<Size_T N = VarSize, Parallel_T parQ = Sequential, Op opx = Op::Id, Op opy = Op::Id,
        typename S, typename T, typename I = Size_T>
    inline auto dot_buffers( const S * x, const T * y, const I n = static_cast<I>(N), const Size_T = 1 )
    {
        using R = decltype( S(0) * T(0) );
        const Size_T m = (N > VarSize) ? N : static_cast<Size_T>(n);
        R r = R(0);
        for( Size_T i = 0; i < m; ++i ) { r += opval<opx>( static_cast<R>(x[i]) ) * opval<opy>( static_cast<R>(y[i]) ); }
        return r;
    }

    template<typename T, typename I>
    inline bool buffers_equalQ( const T * a, const T * b, const I n )
    {
        for( I i = 0; i < n; ++i ) { if( !(a[i] == b[i]) ) { return false; } }
        return true;
    }

    // Inclusive prefix sum in place.
    template<Parallel_T parQ = Sequential, typename T, typename I, typename J = Size_T>
    inline void Accumulate( T * a, const I n, const J = 1 )
    {
        for( I i = 1; i < n; ++i ) { a[i] += a[i-1]; }
    }

    template<typename Iter, typename Comp = std::less<>>
    inline void Sort( Iter begin, Iter end, Comp comp = Comp() )
    {
        std::sort( begin, end, comp );
    }

    // ---------------------------------------------------------------- caching
    // Key-value cache that const methods may fill (mutable storage).
    template<int A_ = 1, int B_ = 1, int C_ = 1, int D_ = 1>
    class CachedObject
    {
    protected:
        mutable std::map<std::string,std::any> cache;
        mutable std::map<std::string,std::any> persistent_cache;
    public:
        CachedObject() = default;
        virtual ~CachedObject() = default;
        CachedObject( const CachedObject & ) = default;
        CachedObject & operator=( const CachedObject & ) = default;
        CachedObject( CachedObject && ) = default;
        CachedObject & operator=( CachedObject && ) = default;

        void ClearCache() const { cache.clear(); }
        void ClearPersistentCache() const { persistent_cache.clear(); }
        bool InCacheQ( const std::string & key ) const { return cache.count(key) > 0; }
        bool InPersistentCacheQ( const std::string & key ) const { return persistent_cache.count(key) > 0; }
        void SetCache( const std::string & key, std::any && v ) const { cache[key] = std::move(v); }
        void SetPersistentCache( const std::string & key, std::any && v ) const { persistent_cache[key] = std::move(v); }
        template<typename T> const T & GetCache( const std::string & key ) const
        {
            return std::any_cast<const T &>( cache.at(key) );
        }
        template<typename T> const T & GetPersistentCache( const std::string & key ) const
        {
            return std::any_cast<const T &>( persistent_cache.at(key) );
        }
    };

} // namespace Tools
