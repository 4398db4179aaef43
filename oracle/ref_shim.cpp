// ref_shim.cpp -- runs the reference's OpenCL kernels on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.py compiles this file together
// with the reference's own kernel source
// (spikesorting_fullpursuit/kernels/binary_pursuit.cl, read where it lies and
// never copied into the repository) into oracle/_ref/libbp_ref.so.  The
// library is driven by the reference's unmodified host function through
// oracle/fake_pyopencl.py to produce the golden vectors under tests/golden/,
// and times the reference kernels for the CPU baseline of bench.py.
//
// OpenCL C is compiled as C++ through the macros below.  A work-group runs on
// one OS thread.  Kernels that call barrier() run each work-item as a fiber;
// the scheduler resumes the fibers of a group in ascending local id until each
// reaches the next barrier, so barrier semantics (and the reference's tie
// order in max_local_reduction, binary_pursuit.cl:167-186) are exact.
// Kernels whose work-items race on shared state in the reference
// (compute_residual, check_overlap_reassignments, binary_pursuit) run their
// work-groups in order on one thread: that fixes the canonical order.
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define __kernel static
#define __global
#define __local
#define __private
#define __constant const
#define restrict __restrict__
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

namespace {

struct WorkItem {
    size_t gid, lid, lsize, gsize;
};

thread_local WorkItem* tl_item = nullptr;
thread_local uint32_t tl_group_slot[16];

inline size_t get_global_id(unsigned) { return tl_item->gid; }
inline size_t get_local_id(unsigned) { return tl_item->lid; }
inline size_t get_local_size(unsigned) { return tl_item->lsize; }
inline size_t get_global_size(unsigned) { return tl_item->gsize; }
inline unsigned int atomic_add(unsigned int* p, unsigned int v)
{
    return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
// The one kernel-scope __local variable (binary_pursuit.cl:968) is rewritten
// by build_ref.py into a reference to this per-group slot.
inline unsigned int* clshim_group_u32() { return &tl_group_slot[0]; }
void barrier(int);

}  // namespace

#include "binary_pursuit_ref.inc"

// ---------------------------------------------------------------------------
// Fibers: x86-64 System V context switch (callee-saved registers only).
// ---------------------------------------------------------------------------
#if defined(__x86_64__)
extern "C" void clshim_switch(void** save_sp, void* load_sp);
asm(R"(
.text
.globl clshim_switch
.type clshim_switch,@function
clshim_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
.size clshim_switch,.-clshim_switch
)");
#else
#error "ref_shim.cpp: fiber switch implemented for x86-64 only"
#endif

namespace {

typedef void (*item_fn)(void** args);

struct Fiber {
    void* sp;
    char* stack;
    bool done;
    WorkItem item;
};

constexpr size_t kStack = 64 * 1024;

thread_local void* tl_sched_sp = nullptr;
thread_local Fiber* tl_fiber = nullptr;
thread_local item_fn tl_fn = nullptr;
thread_local void** tl_args = nullptr;
thread_local std::vector<Fiber>* tl_fibers = nullptr;

[[noreturn]] void fiber_entry()
{
    tl_fn(tl_args);
    tl_fiber->done = true;
    clshim_switch(&tl_fiber->sp, tl_sched_sp);
    __builtin_unreachable();
}

void barrier(int)
{
    if (tl_fiber) clshim_switch(&tl_fiber->sp, tl_sched_sp);
}

void fiber_reset(Fiber& f)
{
    uintptr_t top = (reinterpret_cast<uintptr_t>(f.stack) + kStack) & ~static_cast<uintptr_t>(15);
    void** sp = reinterpret_cast<void**>(top);
    *--sp = nullptr;                                  // alignment slot
    *--sp = reinterpret_cast<void*>(&fiber_entry);    // return target of the first switch
    for (int i = 0; i < 6; ++i) *--sp = nullptr;      // rbp rbx r12 r13 r14 r15
    f.sp = sp;
    f.done = false;
}

std::vector<Fiber>& fibers_for(size_t n)
{
    if (!tl_fibers) tl_fibers = new std::vector<Fiber>();
    while (tl_fibers->size() < n) {
        Fiber f{};
        f.stack = static_cast<char*>(std::malloc(kStack));
        tl_fibers->push_back(f);
    }
    return *tl_fibers;
}

// Runs one work-group whose work-items may call barrier().
void run_group_fibers(item_fn fn, void** args, size_t group, size_t lsize, size_t goff, size_t gsize)
{
    std::vector<Fiber>& fs = fibers_for(lsize);
    for (size_t i = 0; i < lsize; ++i) {
        fiber_reset(fs[i]);
        fs[i].item = WorkItem{goff + group * lsize + i, i, lsize, gsize};
    }
    tl_fn = fn;
    tl_args = args;
    bool any = true;
    while (any) {
        any = false;
        for (size_t i = 0; i < lsize; ++i) {
            if (fs[i].done) continue;
            tl_fiber = &fs[i];
            tl_item = &fs[i].item;
            clshim_switch(&tl_sched_sp, fs[i].sp);
            if (!fs[i].done) any = true;
        }
    }
    tl_fiber = nullptr;
    tl_item = nullptr;
}

// Runs one work-group whose work-items never call barrier().
void run_group_plain(item_fn fn, void** args, size_t group, size_t lsize, size_t goff, size_t gsize)
{
    WorkItem it{0, 0, lsize, gsize};
    tl_item = &it;
    for (size_t i = 0; i < lsize; ++i) {
        it.gid = goff + group * lsize + i;
        it.lid = i;
        fn(args);
    }
    tl_item = nullptr;
}

#define U32(i) (*static_cast<const unsigned int*>(a[i]))
#define PTR(T, i) (static_cast<T*>(a[i]))

void k_compute_residual(void** a)
{
    compute_residual(PTR(float, 0), U32(1), U32(2), PTR(const float, 3), U32(4), U32(5),
                     PTR(const unsigned int, 6), PTR(const unsigned int, 7), U32(8));
}
void k_compute_full_likelihood(void** a)
{
    compute_full_likelihood(PTR(float, 0), U32(1), U32(2), PTR(const float, 3), U32(4), U32(5),
                            PTR(const float, 6), PTR(const unsigned int, 7), U32(8), PTR(float, 9));
}
void k_compute_template_maximum_likelihood(void** a)
{
    compute_template_maximum_likelihood(U32(0), U32(1), U32(2), PTR(const unsigned int, 3), U32(4),
                                        PTR(unsigned int, 5), PTR(unsigned int, 6), PTR(float, 7),
                                        PTR(unsigned char, 8), PTR(unsigned char, 9),
                                        PTR(unsigned int, 10), PTR(unsigned int, 11), PTR(float, 12),
                                        PTR(const float, 13));
}
void k_overlap_recheck_indices(void** a)
{
    overlap_recheck_indices(PTR(float, 0), U32(1), U32(2), PTR(const float, 3), U32(4), U32(5),
                            PTR(const unsigned int, 6), U32(7), PTR(unsigned int, 8),
                            PTR(unsigned int, 9), PTR(float, 10), U32(11), PTR(float, 12),
                            PTR(unsigned int, 13), PTR(float, 14), PTR(unsigned int, 15),
                            PTR(const float, 16));
}
void k_parse_overlap_recheck_indices(void** a)
{
    parse_overlap_recheck_indices(U32(0), U32(1), PTR(const unsigned int, 2), U32(3),
                                  PTR(unsigned int, 4), PTR(unsigned int, 5), PTR(float, 6),
                                  PTR(unsigned int, 7), PTR(unsigned int, 8), PTR(float, 9), U32(10),
                                  PTR(const float, 11), PTR(float, 12), PTR(unsigned int, 13),
                                  PTR(unsigned char, 14));
}
void k_check_overlap_reassignments(void** a)
{
    check_overlap_reassignments(U32(0), U32(1), PTR(const unsigned int, 2), U32(3),
                                PTR(unsigned int, 4), PTR(unsigned int, 5), PTR(unsigned char, 6),
                                PTR(unsigned int, 7), PTR(unsigned int, 8), PTR(unsigned char, 9));
}
void k_binary_pursuit(void** a)
{
    binary_pursuit(U32(0), U32(1), U32(2), PTR(const float, 3), PTR(unsigned int, 4), U32(5),
                   PTR(const unsigned int, 6), PTR(const unsigned int, 7), PTR(const float, 8),
                   PTR(unsigned int, 9), PTR(unsigned int, 10), PTR(unsigned int, 11),
                   PTR(unsigned int, 12), PTR(unsigned char, 13), PTR(unsigned char, 14));
}
void k_get_adjusted_clips(void** a)
{
    get_adjusted_clips(PTR(const float, 0), U32(1), U32(2), PTR(const float, 3), U32(4), U32(5),
                       PTR(const unsigned int, 6), PTR(const unsigned int, 7), U32(8), PTR(float, 9));
}

struct KernelInfo {
    const char* name;
    item_fn fn;
    int nargs;
    bool barriers;     // work-items call barrier()
    bool sequential;   // work-groups run in order on one thread
};

const KernelInfo kKernels[] = {
    {"compute_residual", k_compute_residual, 9, false, true},
    {"compute_full_likelihood", k_compute_full_likelihood, 10, false, false},
    {"compute_template_maximum_likelihood", k_compute_template_maximum_likelihood, 14, false, false},
    {"overlap_recheck_indices", k_overlap_recheck_indices, 17, true, false},
    {"parse_overlap_recheck_indices", k_parse_overlap_recheck_indices, 15, false, false},
    {"check_overlap_reassignments", k_check_overlap_reassignments, 10, false, true},
    {"binary_pursuit", k_binary_pursuit, 15, true, true},
    {"get_adjusted_clips", k_get_adjusted_clips, 10, false, false},
};

}  // namespace

// Argument descriptor: kind 0 = global buffer (ptr is the buffer address),
// 1 = scalar (ptr points at the value), 2 = __local memory of `size` bytes.
struct clshim_arg {
    int32_t kind;
    uint64_t size;
    void* ptr;
};

extern "C" int clshim_nargs(const char* name)
{
    for (const KernelInfo& k : kKernels)
        if (std::strcmp(k.name, name) == 0) return k.nargs;
    return -1;
}

extern "C" int clshim_launch(const char* name, int nargs, const clshim_arg* args, uint64_t goff,
                             uint64_t gsize, uint64_t lsize, int threads)
{
    const KernelInfo* K = nullptr;
    for (const KernelInfo& k : kKernels)
        if (std::strcmp(k.name, name) == 0) K = &k;
    if (!K || nargs != K->nargs || lsize == 0 || gsize % lsize != 0) return -1;
    const int64_t ngroups = static_cast<int64_t>(gsize / lsize);
    int nth = threads > 0 ? threads : 1;
    if (K->sequential) nth = 1;
#pragma omp parallel num_threads(nth)
    {
        // private argument vector: __local arguments get per-thread storage
        std::vector<void*> a(nargs);
        std::vector<std::vector<unsigned char>> locals(nargs);
        for (int i = 0; i < nargs; ++i) {
            if (args[i].kind == 2) {
                locals[i].assign(args[i].size + 64, 0);
                a[i] = locals[i].data();
            } else {
                a[i] = args[i].ptr;
            }
        }
#pragma omp for schedule(dynamic, 1)
        for (int64_t g = 0; g < ngroups; ++g) {
            if (K->barriers)
                run_group_fibers(K->fn, a.data(), static_cast<size_t>(g), lsize, goff, gsize);
            else
                run_group_plain(K->fn, a.data(), static_cast<size_t>(g), lsize, goff, gsize);
        }
    }
    return 0;
}
