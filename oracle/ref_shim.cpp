// ref_shim.cpp -- exposes the reference's own CPU implementations through a
// C ABI so tests can pin the oracle against them and bench.py can time them.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from
// the reference's headers where they lie (cuda_code/SeqMdiscr.h,
// cuda_code/OpenmpMdiscr.h, cuda_code/HelpersCommon.h); nothing of the
// reference is copied here.  The product never loads this library.
//
// What this file adds around the reference headers:
//  * ShimTuple<N>: the reference's OpenmpMdiscr.h:32,38 constructs
//    `TupleType(0)`, a constructor that MyInt4/MyInt8/MyInt<N>
//    (HelpersCommon.h:406-1198) lack, so the OpenMP path only compiles with a
//    tuple type that has one.  ShimTuple<N> is that minimal type.
//  * RecMod<N>: an 8-byte record {u32 key, u32 payload} discriminator with
//    apply = key % N, the semantics of ModArray<N,2> (MdiscrHost_arrays.cu.h:26-36)
//    expressed as an InType the reference's seqMdiscr accepts directly.
//  * stdout capture: both reference routines print their own runtime
//    (SeqMdiscr.h:50-55, OpenmpMdiscr.h:73-76); the shim captures that line
//    and returns the microseconds so callers can report the reference's own
//    timer.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <unistd.h>

#include "HelpersCommon.h"   // Mod4, Mod8, Mod<N>, MyInt*, seqMdiscr (via SeqMdiscr.h)
#include "OpenmpMdiscr.h"    // openmpMdiscr<DISCR>

namespace {

template <unsigned N>
struct ShimTuple {
    unsigned int arr[N];
    static const unsigned int cardinal = N;
    ShimTuple() { for (unsigned i = 0; i < N; i++) arr[i] = 0; }
    explicit ShimTuple(int v) { for (unsigned i = 0; i < N; i++) arr[i] = (unsigned)v; }
    unsigned int& operator[](unsigned i) { return arr[i]; }
    const unsigned int& operator[](unsigned i) const { return arr[i]; }
    friend ShimTuple operator+(const ShimTuple& a, const ShimTuple& b) {
        ShimTuple r;
        for (unsigned i = 0; i < N; i++) r.arr[i] = a.arr[i] + b.arr[i];
        return r;
    }
};

template <unsigned N>
struct ShimMod {                       // Mod<N> with a tuple OpenmpMdiscr can build
    typedef unsigned int InType;
    typedef ShimTuple<N> TupleType;
    static const InType padelm = N - 1;
    static inline unsigned int apply(InType x) { return x % N; }
};

struct Rec { unsigned int key; unsigned int payload; };

template <unsigned N>
struct RecMod {                        // ModArray<N,2>: class from the first word
    typedef Rec InType;
    typedef MyInt<N> TupleType;
    static inline unsigned int apply(const InType& x) { return x.key % N; }
};

// Runs f() with fd 1 redirected to a temporary file; returns the integer that
// follows "runtime:" in what was printed, or -1.
template <class F>
long capture_runtime_us(F f) {
    fflush(stdout);
    FILE* tmp = tmpfile();
    int saved = dup(1);
    if (tmp && saved >= 0) dup2(fileno(tmp), 1);
    f();
    fflush(stdout);
    long us = -1;
    if (tmp && saved >= 0) {
        dup2(saved, 1);
        close(saved);
        rewind(tmp);
        char line[256];
        while (fgets(line, sizeof line, tmp)) {
            const char* p = strstr(line, "runtime:");
            if (p) us = strtol(p + 8, nullptr, 10);
        }
        fclose(tmp);
    }
    return us;
}

template <class D>
long seq_run(unsigned n, void* in, void* out, unsigned* headflags, int measure) {
    typedef typename D::InType T;
    if (measure)
        return capture_runtime_us([&] { seqMdiscr<D, true>(n, (T*)in, (T*)out, headflags); });
    seqMdiscr<D, false>(n, (T*)in, (T*)out, headflags);
    return 0;
}

}  // namespace

// The m values each entry point is instantiated for; anything else returns -2.
#define REF_M_LIST(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(16) X(32) X(64)

extern "C" {

// seqMdiscr<Mod<m>> on n u32 values.  headflags must hold n+1 entries: the
// reference writes one past the end when trailing classes are empty.
// `specialized` selects Mod4 / Mod8 (MyInt4 / MyInt8 tuples) for m = 4 / 8.
long ref_seq_mdiscr_u32(unsigned m, unsigned n, const unsigned* in, unsigned* out,
                        unsigned* headflags, int specialized, int measure) {
    void* vin = const_cast<unsigned*>(in);
    if (specialized && m == 4) return seq_run<Mod4>(n, vin, out, headflags, measure);
    if (specialized && m == 8) return seq_run<Mod8>(n, vin, out, headflags, measure);
#define X(M) if (m == M) return seq_run<Mod<M>>(n, vin, out, headflags, measure);
    REF_M_LIST(X)
#undef X
    return -2;
}

// seqMdiscr over 8-byte records {key, payload}, class = key % m.
long ref_seq_mdiscr_rec8(unsigned m, unsigned n, const void* in, void* out,
                         unsigned* headflags, int measure) {
    void* vin = const_cast<void*>(in);
#define X(M) if (m == M) return seq_run<RecMod<M>>(n, vin, out, headflags, measure);
    REF_M_LIST(X)
#undef X
    return -2;
}

// openmpMdiscr<Mod<m>> on n u32 values; returns the reference's own timer in
// microseconds.  Threads come from OMP_NUM_THREADS / omp_set_num_threads.
long ref_openmp_mdiscr_u32(unsigned m, unsigned n, const unsigned* in, unsigned* out,
                           int* headflags, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    unsigned* vin = const_cast<unsigned*>(in);
#define X(M) if (m == M) return capture_runtime_us([&] { openmpMdiscr<ShimMod<M>>(n, vin, out, headflags); });
    REF_M_LIST(X)
#undef X
    return -2;
}

int ref_openmp_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
