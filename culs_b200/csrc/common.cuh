// Shared device helpers: status word, bounded waits, atomics, literal helpers.
//
// Kernel bodies are written as __host__ __device__ functions over plain
// arrays so that their logic can be exercised one item at a time; the
// atomics and memory-order helpers below map to the CUDA intrinsics in device
// code and to plain sequential operations in host code.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define CULS_HD __host__ __device__ __forceinline__
#define CULS_DEV __device__ __forceinline__
#else
#define CULS_HD inline
#define CULS_DEV inline
#endif

namespace culs {

// ----------------------------------------------------------- status codes
// Written into the context's device status word by the first failing thread;
// the host maps it to a CULS_E_* code after each stage.
enum DevStatus : int32_t {
    kDevOk = 0,
    kDevWaitTimeout = 1,   // a bounded dependency wait expired
    kDevTableFull = 2,     // a hash table probe sequence hit its cap
    kDevStackOverflow = 3, // an explicit traversal stack overflowed
    kDevBadGraph = 4,      // structural inconsistency (cycle, bad literal)
    kDevCapacity = 5,      // a work buffer was too small
    kDevAigerFormat = 6,   // binary AIGER bytes do not decode
};

// Upper bound on spin iterations of a dependency wait (each iteration sleeps
// up to 256 ns after the first 64): about one second.
constexpr int64_t kSpinLimit = 1ll << 22;

CULS_HD int lit_id(int lit) { return lit >> 1; }
CULS_HD int lit_c(int lit) { return lit & 1; }

// -------------------------------------------------------------- atomics
#if defined(__CUDA_ARCH__)
CULS_DEV int at_add(int *p, int v) { return atomicAdd(p, v); }
CULS_DEV unsigned long long at_add(unsigned long long *p, unsigned long long v) { return atomicAdd(p, v); }
CULS_DEV int at_min(int *p, int v) { return atomicMin(p, v); }
CULS_DEV unsigned long long at_min(unsigned long long *p, unsigned long long v) { return atomicMin(p, v); }
CULS_DEV int at_cas(int *p, int cmp, int v) { return atomicCAS(p, cmp, v); }
CULS_DEV unsigned long long at_cas(unsigned long long *p, unsigned long long cmp, unsigned long long v) {
    return atomicCAS(p, cmp, v);
}
CULS_DEV int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
CULS_DEV void st_release(int *p, int v) { asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }
// Relaxed GPU-scope accesses, for a word that is itself the published value
// (a level): the reader uses nothing else the writer stored before it, so
// coherence of the one word is all the ordering needed.
CULS_DEV int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
CULS_DEV void st_relaxed(int *p, int v) { asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }
CULS_DEV int ld_cg(const int *p) { return __ldcg(p); }
CULS_DEV int4 ld_cg(const int4 *p) { return __ldcg(p); }
CULS_DEV int2 ld_cg(const int2 *p) { return __ldcg(p); }
CULS_DEV void set_status(int *status, int code) { atomicCAS(status, 0, code); }
CULS_DEV void backoff(int64_t it) {
    if (it > 64) __nanosleep(it > 4096 ? 256 : 64);
}
#else
inline int at_add(int *p, int v) {
    int o = *p;
    *p += v;
    return o;
}
inline unsigned long long at_add(unsigned long long *p, unsigned long long v) {
    unsigned long long o = *p;
    *p += v;
    return o;
}
inline int at_min(int *p, int v) {
    int o = *p;
    if (v < o) *p = v;
    return o;
}
inline unsigned long long at_min(unsigned long long *p, unsigned long long v) {
    unsigned long long o = *p;
    if (v < o) *p = v;
    return o;
}
inline int at_cas(int *p, int cmp, int v) {
    int o = *p;
    if (o == cmp) *p = v;
    return o;
}
inline unsigned long long at_cas(unsigned long long *p, unsigned long long cmp, unsigned long long v) {
    unsigned long long o = *p;
    if (o == cmp) *p = v;
    return o;
}
inline int ld_acquire(const int *p) { return *p; }
inline void st_release(int *p, int v) { *p = v; }
inline int ld_relaxed(const int *p) { return *p; }
inline void st_relaxed(int *p, int v) { *p = v; }
inline int ld_cg(const int *p) { return *p; }
inline void set_status(int *status, int code) {
    if (*status == 0) *status = code;
}
inline void backoff(int64_t) {}
#endif

// A status pointer handed to a kernel addresses two words: status[0] is the
// status word the first failing thread writes, status[1] the spin bound of
// the dependency waits that report into it (0 means kSpinLimit).  The host
// lowers the bound (CULS_SPIN_LIMIT) to make waits run out on purpose.
CULS_HD int64_t spin_limit(const int *status) {
    const int l = ld_cg(status + 1);
    return l > 0 ? (int64_t)l : kSpinLimit;
}

// Waits until *flag >= target.  Returns false (and records kDevWaitTimeout)
// when the bound expires, so that no dependency wait can hang the GPU.  A
// wait also gives up at once, without recording anything, when the status
// word already holds an error: the call has failed, and the work it waits
// for may itself have been skipped, so one expired wait does not make every
// dependent wait spin out its own bound.
CULS_HD bool wait_ge(const int *flag, int target, int *status) {
    if (ld_acquire(flag) >= target) return true;
    const int64_t lim = spin_limit(status);
    for (int64_t it = 1;; ++it) {
        if ((it & 31) == 1 && ld_cg(status) != kDevOk) return false;
        if (it >= lim) {
            set_status(status, kDevWaitTimeout);
            return false;
        }
        backoff(it);
        if (ld_acquire(flag) >= target) return true;
    }
}

// Waits until the word *w is at least `floor` and returns it in *val: the
// same bounds as wait_ge, with relaxed loads, for a word that carries its
// own payload (see ld_relaxed).
CULS_HD bool wait_word(const int *w, int floor, int *status, int *val) {
    int v = ld_relaxed(w);
    if (v >= floor) {
        *val = v;
        return true;
    }
    const int64_t lim = spin_limit(status);
    for (int64_t it = 1;; ++it) {
        if ((it & 31) == 1 && ld_cg(status) != kDevOk) return false;
        if (it >= lim) {
            set_status(status, kDevWaitTimeout);
            return false;
        }
        backoff(it);
        v = ld_relaxed(w);
        if (v >= floor) {
            *val = v;
            return true;
        }
    }
}

// MurmurHash3 64-bit finalizer (public domain, Austin Appleby).
CULS_HD uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

constexpr unsigned long long kEmptyKey = ~0ull;

}  // namespace culs
