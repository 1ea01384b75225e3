// CPU stand-in for the subset of SYCL 2020 that MacraMacra/OS2-Xe's src/ozaki2_gpu.hpp and
// tests/test_ozaki2.cpp use, so that the reference's own sources compile with g++ and run on
// the host as the oracle's cross-check (oracle/_ref). TEST INFRASTRUCTURE ONLY.
//
// Execution model: every submit runs synchronously on the calling thread's OpenMP team.
// range<> kernels are plain loops; nd_range<> work-groups run their work-items as ucontext
// coroutines so that group_barrier / reduce_over_group have real barrier semantics.
#pragma once

#include <ucontext.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace sycl {

// ---------------------------------------------------------------- scalar built-ins
template <class To, class From>
inline To bit_cast(const From& f) {
    static_assert(sizeof(To) == sizeof(From), "bit_cast size");
    To t;
    std::memcpy(&t, &f, sizeof t);
    return t;
}
inline uint32_t mul_hi(uint32_t a, uint32_t b) { return static_cast<uint32_t>((uint64_t{a} * b) >> 32); }
template <class T> inline T min(T a, T b) { return b < a ? b : a; }
template <class T> inline T max(T a, T b) { return a < b ? b : a; }
inline float fma(float a, float b, float c) { return std::fma(a, b, c); }
inline double fma(double a, double b, double c) { return std::fma(a, b, c); }
inline float rint(float x) { return std::rint(x); }
inline double rint(double x) { return std::rint(x); }
inline uint32_t clz(uint32_t x) { return x ? static_cast<uint32_t>(__builtin_clz(x)) : 32u; }
inline double ldexp(double x, int e) { return std::ldexp(x, e); }
inline double sin(double x) { return std::sin(x); }
inline double cos(double x) { return std::cos(x); }
inline double sqrt(double x) { return std::sqrt(x); }
inline double log(double x) { return std::log(x); }
inline double exp(double x) { return std::exp(x); }
inline double fabs(double x) { return std::fabs(x); }
template <class T>
struct private_ptr {
    T* p;
    explicit private_ptr(T* q) : p(q) {}
};
inline double frexp(double x, private_ptr<int> e) { return std::frexp(x, e.p); }

// ---------------------------------------------------------------- index space
template <int D>
struct range {
    size_t v[D];
    range(size_t a) : v{a} { static_assert(D == 1, "range<1>"); }
    range(size_t a, size_t b) : v{a, b} { static_assert(D == 2, "range<2>"); }
    size_t operator[](int i) const { return v[i]; }
    size_t size() const {
        size_t s = 1;
        for (int i = 0; i < D; ++i) s *= v[i];
        return s;
    }
};
template <int D>
struct id {
    size_t v[D];
    size_t operator[](int i) const { return v[i]; }
};
template <>
struct id<1> {
    size_t v[1];
    size_t operator[](int i) const { return v[i]; }
    operator size_t() const { return v[0]; }
};
template <int D>
struct nd_range {
    range<D> g, l;
    nd_range(range<D> gg, range<D> ll) : g(gg), l(ll) {}
};

template <class T>
struct maximum {
    T operator()(const T& a, const T& b) const { return a < b ? b : a; }
};

// ---------------------------------------------------------------- work-group runtime
namespace detail {
constexpr size_t kStack = 64 * 1024;

struct GroupRun {
    int n = 0;              // work-items in the group
    int cur = 0;            // running item
    bool coro = false;      // items run as coroutines
    bool yielded = false;   // the probe item hit a group operation
    bool reducing = false;  // the pending group operation is a reduction
    std::vector<ucontext_t> ctx;
    std::vector<char> stacks;
    std::vector<int> state; // 0 ready, 1 at barrier, 2 done
    std::vector<unsigned char> slots;
    unsigned char result[16];
    ucontext_t sched;
    void (*fn)(void*, int) = nullptr;
    void* obj = nullptr;
    std::vector<unsigned char> local; // local memory of this group
};
inline GroupRun*& tls_run() {
    static thread_local GroupRun* r = nullptr;
    return r;
}
inline void trampoline() {
    GroupRun* r = tls_run();
    const int me = r->cur;
    r->fn(r->obj, me);
    r->state[me] = 2;
    // returning resumes r->sched through uc_link
}
inline void yield_to_sched() {
    GroupRun* r = tls_run();
    swapcontext(&r->ctx[r->cur], &r->sched);
}
inline void fatal(const char* what) {
    std::fprintf(stderr, "sycl stand-in: %s\n", what);
    std::abort();
}
}  // namespace detail

struct group {};

template <class T, class Op>
inline T reduce_over_group(group, T x, Op op) {
    static_assert(sizeof(T) <= 16, "reduce type");
    detail::GroupRun* r = detail::tls_run();
    if (!r || !r->coro) detail::fatal("group operation outside a coroutine work-group");
    if (r->slots.size() < static_cast<size_t>(r->n) * 16) r->slots.resize(static_cast<size_t>(r->n) * 16);
    std::memcpy(&r->slots[static_cast<size_t>(r->cur) * 16], &x, sizeof(T));
    r->reducing = true;
    r->state[r->cur] = 1;
    r->yielded = true;
    detail::yield_to_sched();
    T out;
    std::memcpy(&out, r->result, sizeof(T));
    (void)op;
    return out;
}
template <class T>
inline T group_reduce_combine(const std::vector<unsigned char>& slots, int n, maximum<T> op) {
    T acc;
    std::memcpy(&acc, &slots[0], sizeof(T));
    for (int i = 1; i < n; ++i) {
        T v;
        std::memcpy(&v, &slots[static_cast<size_t>(i) * 16], sizeof(T));
        acc = op(acc, v);
    }
    return acc;
}
inline void group_barrier(group) {
    detail::GroupRun* r = detail::tls_run();
    if (!r || !r->coro) detail::fatal("group_barrier outside a coroutine work-group");
    r->state[r->cur] = 1;
    r->yielded = true;
    detail::yield_to_sched();
}

template <int D>
struct nd_item {
    size_t gid[D], lid[D], grp[D];
    size_t get_global_id(int d) const { return gid[d]; }
    size_t get_local_id(int d) const { return lid[d]; }
    size_t get_group(int d) const { return grp[d]; }
    group get_group() const { return group{}; }
};

// ---------------------------------------------------------------- memory model
enum class memory_order { relaxed, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, private_space, generic_space };
}
template <class T, memory_order MO, memory_scope MS, access::address_space AS = access::address_space::generic_space>
struct atomic_ref {
    T& ref;
    explicit atomic_ref(T& r) : ref(r) {}
    T fetch_max(T v) const {
        T old = __atomic_load_n(&ref, __ATOMIC_RELAXED);
        while (old < v && !__atomic_compare_exchange_n(&ref, &old, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
        }
        return old;
    }
};

// ---------------------------------------------------------------- properties / device / event
namespace property {
namespace queue {
struct in_order {};
struct enable_profiling {};
}  // namespace queue
}  // namespace property
struct property_list {
    bool profiling = false;
    property_list() = default;
    template <class... P>
    property_list(P... ps) {
        profiling = (std::is_same_v<P, property::queue::enable_profiling> || ...);
    }
};
struct gpu_selector_t {};
inline constexpr gpu_selector_t gpu_selector_v{};

namespace info {
namespace device {
struct name { using return_type = std::string; static std::string get() { return "oz2 CPU stand-in for SYCL"; } };
struct global_mem_size { using return_type = size_t; static size_t get() { return size_t{64} << 30; } };
struct max_mem_alloc_size { using return_type = size_t; static size_t get() { return size_t{64} << 30; } };
}  // namespace device
namespace event_profiling {
struct command_start {};
struct command_end {};
}  // namespace event_profiling
}  // namespace info
namespace ext {
namespace intel {
namespace info {
namespace device {
struct free_memory { using return_type = size_t; static size_t get() { return size_t{60} << 30; } };
}  // namespace device
}  // namespace info
}  // namespace intel
}  // namespace ext

struct device {
    template <class P>
    typename P::return_type get_info() const { return P::get(); }
};

struct event {
    uint64_t t0 = 0, t1 = 0;
    void wait() const {}
    template <class P>
    uint64_t get_profiling_info() const {
        return std::is_same_v<P, info::event_profiling::command_start> ? t0 : t1;
    }
};
inline uint64_t now_ns() {
    return static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
            .count());
}

// ---------------------------------------------------------------- handler
class handler;
template <class V, int D>
struct local_accessor {
    size_t off = 0;
    size_t dim1 = 1;
    local_accessor(range<D> r, handler& h);
    V* operator[](size_t a) const {
        detail::GroupRun* g = detail::tls_run();
        return reinterpret_cast<V*>(g->local.data() + off) + a * dim1;
    }
};

class handler {
public:
    size_t local_bytes = 0;
    void depends_on(const event&) {}
    void depends_on(const std::vector<event>&) {}

    template <class F>
    void parallel_for(range<1> r, F f) {
        const int64_t n = static_cast<int64_t>(r[0]);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) f(id<1>{{static_cast<size_t>(i)}});
    }
    template <class F>
    void parallel_for(range<2> r, F f) {
        const int64_t n0 = static_cast<int64_t>(r[0]), n1 = static_cast<int64_t>(r[1]);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n0; ++i)
            for (int64_t j = 0; j < n1; ++j) f(id<2>{{static_cast<size_t>(i), static_cast<size_t>(j)}});
    }
    template <int D, class F>
    void parallel_for(nd_range<D> nr, F f) {
        size_t G[2] = {1, 1}, L[2] = {1, 1};
        for (int d = 0; d < D; ++d) {
            if (nr.g[d] % nr.l[d]) detail::fatal("nd_range global size not a multiple of the local size");
            G[d] = nr.g[d] / nr.l[d];
            L[d] = nr.l[d];
        }
        const int64_t groups = static_cast<int64_t>(G[0] * G[1]);
        const int items = static_cast<int>(L[0] * L[1]);
        const size_t lb = local_bytes;
#pragma omp parallel
        {
            detail::GroupRun run;
            run.n = items;
            run.local.assign(lb, 0);
            detail::tls_run() = &run;
            struct Ctx {
                F* f;
                size_t g[2], L[2];
            } ctx{&f, {0, 0}, {L[0], L[1]}};
            run.obj = &ctx;
            run.fn = [](void* o, int li) {
                Ctx* c = static_cast<Ctx*>(o);
                nd_item<D> it;
                const size_t l[2] = {static_cast<size_t>(li) / c->L[1], static_cast<size_t>(li) % c->L[1]};
                for (int d = 0; d < D; ++d) {
                    it.lid[d] = l[d];
                    it.grp[d] = c->g[d];
                    it.gid[d] = c->g[d] * c->L[d] + l[d];
                }
                (*c->f)(it);
            };
#pragma omp for schedule(dynamic, 4)
            for (int64_t gl = 0; gl < groups; ++gl) {
                ctx.g[0] = static_cast<size_t>(gl) / G[1];
                ctx.g[1] = static_cast<size_t>(gl) % G[1];
                run_group(run);
            }
            detail::tls_run() = nullptr;
        }
    }

private:
    static void start(detail::GroupRun& r, int i) {
        getcontext(&r.ctx[i]);
        r.ctx[i].uc_stack.ss_sp = r.stacks.data() + static_cast<size_t>(i) * detail::kStack;
        r.ctx[i].uc_stack.ss_size = detail::kStack;
        r.ctx[i].uc_link = &r.sched;
        makecontext(&r.ctx[i], detail::trampoline, 0);
        r.state[i] = 0;
    }
    template <class T>
    static void finish_reduce(detail::GroupRun& r) {
        T v = group_reduce_combine<T>(r.slots, r.n, maximum<T>());
        std::memcpy(r.result, &v, sizeof(T));
    }
    static void run_group(detail::GroupRun& r) {
        if (r.ctx.size() < static_cast<size_t>(r.n)) {
            r.ctx.resize(r.n);
            r.stacks.resize(static_cast<size_t>(r.n) * detail::kStack);
        }
        r.state.assign(r.n, 0);
        std::fill(r.local.begin(), r.local.end(), 0);
        // probe: item 0 as a coroutine
        r.coro = true;
        r.yielded = false;
        start(r, 0);
        r.cur = 0;
        swapcontext(&r.sched, &r.ctx[0]);
        if (!r.yielded) {
            r.coro = false;
            for (int i = 1; i < r.n; ++i) {
                r.cur = i;
                r.fn(r.obj, i);
            }
            return;
        }
        for (int i = 1; i < r.n; ++i) start(r, i);
        for (;;) {
            bool any = false;
            for (int i = 0; i < r.n; ++i) {
                if (r.state[i] != 0) continue;
                r.cur = i;
                swapcontext(&r.sched, &r.ctx[i]);
                any = true;
            }
            int done = 0, waiting = 0;
            for (int i = 0; i < r.n; ++i) {
                done += r.state[i] == 2;
                waiting += r.state[i] == 1;
            }
            if (done == r.n) break;
            if (waiting + done == r.n) {
                if (done) detail::fatal("work-items diverged around a group operation");
                // a barrier or a reduction: the only reductions used are maxima of uint64_t
                if (r.reducing) finish_reduce<uint64_t>(r);
                r.reducing = false;
                for (int i = 0; i < r.n; ++i) r.state[i] = 0;
            } else if (!any) {
                detail::fatal("work-group deadlock");
            }
        }
    }
};

template <class V, int D>
local_accessor<V, D>::local_accessor(range<D> r, handler& h) {
    off = (h.local_bytes + 63) / 64 * 64;
    dim1 = D == 2 ? r[1] : 1;
    h.local_bytes = off + r.size() * sizeof(V);
}

// ---------------------------------------------------------------- queue
class queue {
public:
    queue() = default;
    queue(gpu_selector_t, property::queue::in_order) {}
    queue(gpu_selector_t, property_list pl) : profiling_(pl.profiling) {}
    template <class P>
    bool has_property() const {
        return std::is_same_v<P, property::queue::enable_profiling> ? profiling_ : true;
    }
    device get_device() const { return device{}; }
    template <class CGF>
    event submit(CGF cgf) {
        event e;
        e.t0 = now_ns();
        handler h;
        cgf(h);
        e.t1 = now_ns();
        return e;
    }
    template <int D, class F>
    event parallel_for(range<D> r, F f) {
        return submit([&](handler& h) { h.parallel_for(r, f); });
    }
    event memset(void* p, int v, size_t n, event = {}) {
        event e;
        e.t0 = now_ns();
        std::memset(p, v, n);
        e.t1 = now_ns();
        return e;
    }
    event memcpy(void* d, const void* s, size_t n, event = {}) {
        std::memcpy(d, s, n);
        return event{now_ns(), now_ns()};
    }
    event ext_oneapi_submit_barrier(const std::vector<event>& = {}) { return event{now_ns(), now_ns()}; }
    void wait() {}

private:
    bool profiling_ = false;
};

template <class T>
inline T* malloc_device(size_t count, queue&) {
    const size_t bytes = (count * sizeof(T) + 63) / 64 * 64;
    return static_cast<T*>(std::aligned_alloc(64, bytes ? bytes : 64));
}
inline void free(void* p, queue&) { std::free(p); }

}  // namespace sycl
