// template_dropin.cu -- a program written against the reference's host
// templates (mdiscr<DISCR>, mdiscrSegm<DISCR>), compiled against
// include/mdx/mdiscr.cuh instead.  Functors follow the reference's concept:
// InType, TupleType {cardinal, operator[]}, padelm, static apply on the device.
// Each case is checked against a plain CPU stable partition.  Prints one line
// per case and exits non-zero on the first mismatch.  Built with MDX_NO_EXIT,
// so a failing call throws instead of exiting: the first case injects a
// workspace allocation failure (host side) and expects exactly that.
#define MDX_NO_EXIT 1
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "mdx/mdiscr.cuh"

template <unsigned N>
struct Counts {  // tuple of class sizes
    unsigned int arr[N];
    static const unsigned int cardinal = N;
    Counts() { for (unsigned i = 0; i < N; i++) arr[i] = 0; }
    unsigned int& operator[](unsigned i) { return arr[i]; }
};

struct LowBits8 {  // class = x & 7
    typedef unsigned int InType;
    typedef Counts<8> TupleType;
    static const InType padelm = 7;
    __host__ __device__ static inline unsigned int apply(volatile InType x) { return x & 7; }
};

template <unsigned N>
struct Remainder {  // class = x % N
    typedef unsigned int InType;
    typedef Counts<N> TupleType;
    static const InType padelm = N - 1;
    __host__ __device__ static inline unsigned int apply(volatile InType x) { return x % N; }
};

struct Pair {
    unsigned int key, payload;
};
template <unsigned N>
struct KeyRemainder {  // 8-byte records, class = key % N
    typedef Pair InType;
    typedef Counts<N> TupleType;
    __host__ __device__ static inline unsigned int apply(volatile InType x) { return x.key % N; }
};

struct Quad {
    unsigned int key, a, b, c;
};
template <unsigned N>
struct QuadRemainder {  // 16-byte records, class = key % N
    typedef Quad InType;
    typedef Counts<N> TupleType;
    __host__ __device__ static inline unsigned int apply(volatile InType x) { return x.key % N; }
};

struct Decades {  // a functor that is not a remainder: class = (x / 10) % 6
    typedef unsigned int InType;
    typedef Counts<6> TupleType;
    __host__ __device__ static inline unsigned int apply(volatile InType x) { return (x / 10u) % 6u; }
};

template <unsigned N, unsigned LEN>
struct ArrayRemainder {  // records of LEN unsigned ints, class = x[0] % N (ModArray's concept)
    typedef unsigned int InType;
    typedef Counts<N> TupleType;
    static const InType padelm = N - 1;
    __host__ __device__ static inline unsigned int apply(volatile InType* x) { return x[0] % N; }
};

struct MixedTuple {  // (u32, u8, bool) rows, class from all three fields (tuple concept)
    typedef unsigned int InType1;
    typedef unsigned char InType2;
    typedef bool InType3;
    typedef Counts<7> TupleType;
    __host__ __device__ static inline unsigned int apply(volatile InType1 x, volatile InType2 y,
                                                         volatile InType3 z) {
        return z ? x % 7u : y % 7u;
    }
};

static unsigned long long rng_state = 88172645463325252ull;
static unsigned int next_u32() {  // xorshift64
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return static_cast<unsigned int>(rng_state >> 33);
}

template <class D>
static void cpu_partition(const std::vector<typename D::InType>& in, std::vector<typename D::InType>& out,
                          std::vector<unsigned>& sizes, std::vector<int>* flags) {
    const unsigned m = D::TupleType::cardinal;
    sizes.assign(m, 0);
    for (auto& v : in) sizes[D::apply(v)]++;
    std::vector<unsigned> cur(m, 0);
    unsigned acc = 0;
    for (unsigned c = 0; c < m; c++) { cur[c] = acc; acc += sizes[c]; }
    out.resize(in.size());
    for (auto& v : in) out[cur[D::apply(v)]++] = v;
    if (flags) {
        flags->assign(in.size(), 0);
        acc = 0;
        for (unsigned c = 0; c < m; c++) {
            if (sizes[c] && acc < in.size()) (*flags)[acc] = static_cast<int>(sizes[c]);
            acc += sizes[c];
        }
    }
}

template <class D>
static int plain_case(const char* name, unsigned n) {
    typedef typename D::InType T;
    std::vector<T> h(n), want;
    for (unsigned i = 0; i < n; i++) {
        unsigned v[4] = {next_u32(), i, next_u32(), ~i};
        std::memcpy(&h[i], v, sizeof(T));
    }
    std::vector<unsigned> wsz;
    cpu_partition<D>(h, want, wsz, nullptr);
    T *d_in, *d_out;
    cudaMalloc(&d_in, n * sizeof(T) + 1);
    cudaMalloc(&d_out, n * sizeof(T) + 1);
    cudaMemcpy(d_in, h.data(), n * sizeof(T), cudaMemcpyHostToDevice);
    typename D::TupleType sizes = mdiscr<D>(n, 1 << 16, d_in, d_out);
    std::vector<T> got(n);
    cudaMemcpy(got.data(), d_out, n * sizeof(T), cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    bool ok = std::memcmp(got.data(), want.data(), n * sizeof(T)) == 0;
    for (unsigned c = 0; c < D::TupleType::cardinal; c++) ok = ok && sizes[c] == wsz[c];
    std::printf("%s n=%u: %s\n", name, n, ok ? "VALID" : "INVALID");
    return ok ? 0 : 1;
}

template <class D>
static int segm_case(const char* name, unsigned n) {
    typedef typename D::InType T;
    std::vector<T> h(n);
    for (unsigned i = 0; i < n; i++) {
        unsigned v[2] = {next_u32(), i};
        std::memcpy(&h[i], v, sizeof(T));
    }
    std::vector<int> seg(n, 0);  // head-flag segment sizes, lengths 1 .. 20000
    for (unsigned i = 0; i < n;) {
        unsigned len = 1 + next_u32() % (next_u32() % 4 == 0 ? 20000u : 300u);
        if (len > n - i) len = n - i;
        seg[i] = static_cast<int>(len);
        i += len;
    }
    std::vector<T> want(n);
    std::vector<int> wflags(n, 0);
    for (unsigned i = 0; i < n; i += seg[i]) {
        std::vector<T> part(h.begin() + i, h.begin() + i + seg[i]), po;
        std::vector<unsigned> ps;
        std::vector<int> pf;
        cpu_partition<D>(part, po, ps, &pf);
        std::copy(po.begin(), po.end(), want.begin() + i);
        std::copy(pf.begin(), pf.end(), wflags.begin() + i);
    }
    T *d_in, *d_out;
    int *d_seg, *d_new;
    cudaMalloc(&d_in, n * sizeof(T));
    cudaMalloc(&d_out, n * sizeof(T));
    cudaMalloc(&d_seg, n * sizeof(int));
    cudaMalloc(&d_new, n * sizeof(int));
    cudaMemcpy(d_in, h.data(), n * sizeof(T), cudaMemcpyHostToDevice);
    cudaMemcpy(d_seg, seg.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    mdiscrSegm<D>(n, d_in, d_seg, d_out, d_new);
    std::vector<T> got(n);
    std::vector<int> gflags(n);
    cudaMemcpy(got.data(), d_out, n * sizeof(T), cudaMemcpyDeviceToHost);
    cudaMemcpy(gflags.data(), d_new, n * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_seg);
    cudaFree(d_new);
    const bool ok = std::memcmp(got.data(), want.data(), n * sizeof(T)) == 0 && gflags == wflags;
    std::printf("%s n=%u: %s\n", name, n, ok ? "VALID" : "INVALID");
    return ok ? 0 : 1;
}

template <class D, unsigned LEN>
static int array_case(const char* name, unsigned n) {
    const unsigned m = D::TupleType::cardinal;
    std::vector<unsigned> h(static_cast<size_t>(n) * LEN), want(h.size());
    for (auto& v : h) v = next_u32();
    std::vector<unsigned> wsz(m, 0), cur(m, 0);
    for (unsigned i = 0; i < n; i++) wsz[D::apply(&h[static_cast<size_t>(i) * LEN])]++;
    for (unsigned c = 1; c < m; c++) cur[c] = cur[c - 1] + wsz[c - 1];
    for (unsigned i = 0; i < n; i++) {
        const unsigned p = cur[D::apply(&h[static_cast<size_t>(i) * LEN])]++;
        std::memcpy(&want[static_cast<size_t>(p) * LEN], &h[static_cast<size_t>(i) * LEN], LEN * 4);
    }
    unsigned *d_in, *d_out;
    cudaMalloc(&d_in, h.size() * 4);
    cudaMalloc(&d_out, h.size() * 4);
    cudaMemcpy(d_in, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
    typename D::TupleType sizes = mdiscr<D, LEN>(n, 1 << 16, d_in, d_out);
    std::vector<unsigned> got(h.size());
    cudaMemcpy(got.data(), d_out, h.size() * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    bool ok = got == want;
    for (unsigned c = 0; c < m; c++) ok = ok && sizes[c] == wsz[c];
    std::printf("%s n=%u: %s\n", name, n, ok ? "VALID" : "INVALID");
    return ok ? 0 : 1;
}

static int tuple_case(const char* name, unsigned n) {
    typedef MixedTuple D;
    const unsigned m = D::TupleType::cardinal;
    std::vector<unsigned> a(n), wa(n);
    std::vector<unsigned char> b(n), wb(n);
    bool* c = new bool[n];
    bool* wc = new bool[n];
    for (unsigned i = 0; i < n; i++) {
        a[i] = next_u32();
        b[i] = static_cast<unsigned char>(next_u32());
        c[i] = (next_u32() & 1u) != 0;
    }
    std::vector<unsigned> wsz(m, 0), cur(m, 0);
    for (unsigned i = 0; i < n; i++) wsz[D::apply(a[i], b[i], c[i])]++;
    for (unsigned k = 1; k < m; k++) cur[k] = cur[k - 1] + wsz[k - 1];
    for (unsigned i = 0; i < n; i++) {
        const unsigned p = cur[D::apply(a[i], b[i], c[i])]++;
        wa[p] = a[i];
        wb[p] = b[i];
        wc[p] = c[i];
    }
    unsigned *da, *oa;
    unsigned char *db, *ob;
    bool *dc, *oc;
    cudaMalloc(&da, n * 4);
    cudaMalloc(&oa, n * 4);
    cudaMalloc(&db, n);
    cudaMalloc(&ob, n);
    cudaMalloc(&dc, n);
    cudaMalloc(&oc, n);
    cudaMemcpy(da, a.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b.data(), n, cudaMemcpyHostToDevice);
    cudaMemcpy(dc, c, n, cudaMemcpyHostToDevice);
    typename D::TupleType sizes = mdiscr<D>(n, 1 << 16, da, db, dc, oa, ob, oc);
    std::vector<unsigned> ga(n);
    std::vector<unsigned char> gb(n);
    bool* gc = new bool[n];
    cudaMemcpy(ga.data(), oa, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(gb.data(), ob, n, cudaMemcpyDeviceToHost);
    cudaMemcpy(gc, oc, n, cudaMemcpyDeviceToHost);
    cudaFree(da); cudaFree(oa); cudaFree(db); cudaFree(ob); cudaFree(dc); cudaFree(oc);
    bool ok = ga == wa && gb == wb && std::memcmp(gc, wc, n) == 0;
    for (unsigned k = 0; k < m; k++) ok = ok && sizes[k] == wsz[k];
    delete[] c;
    delete[] wc;
    delete[] gc;
    std::printf("%s n=%u: %s\n", name, n, ok ? "VALID" : "INVALID");
    return ok ? 0 : 1;
}

// The first call of the program grows the (empty) workspace; with the
// growth made to fail it must report the failure (std::runtime_error under
// MDX_NO_EXIT) and leave nothing behind, and the next call must succeed.
static int alloc_failure_case() {
    const unsigned n = 100000;
    std::vector<unsigned> h(n);
    for (unsigned i = 0; i < n; i++) h[i] = i * 2654435761u;
    unsigned *d = nullptr, *o = nullptr;
    cudaMalloc(&d, n * 4);
    cudaMalloc(&o, n * 4);
    cudaMemcpy(d, h.data(), n * 4, cudaMemcpyHostToDevice);
    mdx::test_inject_workspace_failure(1);
    bool threw = false;
    try {
        (void)mdiscr<LowBits8>(n, 1024, d, o);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    mdx::test_inject_workspace_failure(0);
    Counts<8> sz = mdiscr<LowBits8>(n, 1024, d, o);  // the workspace grows now
    unsigned total = 0;
    for (unsigned c = 0; c < 8; c++) total += sz[c];
    cudaFree(d);
    cudaFree(o);
    const bool ok = threw && total == n;
    std::printf("workspace allocation failure: %s\n", ok ? "REPORTED" : "NOT REPORTED");
    return ok ? 0 : 1;
}

int main() {
    int bad = 0;
    bad |= alloc_failure_case();
    bad |= plain_case<LowBits8>("mdiscr<LowBits8>", 1u << 20);
    bad |= plain_case<Remainder<5>>("mdiscr<Remainder<5>>", 3000017u);
    bad |= plain_case<Remainder<40>>("mdiscr<Remainder<40>>", 777777u);
    bad |= plain_case<Decades>("mdiscr<Decades>", 100003u);
    bad |= plain_case<KeyRemainder<16>>("mdiscr<KeyRemainder<16>>", 1000003u);
    bad |= plain_case<QuadRemainder<7>>("mdiscr<QuadRemainder<7>>", 654321u);
    bad |= plain_case<QuadRemainder<64>>("mdiscr<QuadRemainder<64>>", 200003u);
    bad |= segm_case<Remainder<4>>("mdiscrSegm<Remainder<4>>", 2000000u);
    bad |= segm_case<KeyRemainder<3>>("mdiscrSegm<KeyRemainder<3>>", 500000u);
    bad |= segm_case<Decades>("mdiscrSegm<Decades>", 300000u);
    bad |= array_case<ArrayRemainder<5, 3>, 3>("mdiscr<ArrayRemainder<5,3>, 3>", 400003u);
    bad |= array_case<ArrayRemainder<16, 8>, 8>("mdiscr<ArrayRemainder<16,8>, 8>", 100000u);
    bad |= tuple_case("mdiscr<MixedTuple>", 500009u);
    return bad;
}
