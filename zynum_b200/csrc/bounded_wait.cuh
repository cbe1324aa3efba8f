// Bounded mbarrier waits shared by the tensor-core kernels (sm_100a).
//
// Every mbarrier wait of the product kernels is bounded in time (%globaltimer,
// nanoseconds).  When one runs out, the waiting role raises the CTA's abort
// flag and records the site in the call's status word (read by the kernels
// that follow on the stream, which then leave C untouched) and in the device's
// report word (read by the host, zynum_blas_gpu_device_status).  The other
// roles of the CTA see the flag within 256 polls and leave their loops; copies
// and MMAs already issued are drained before shared memory and TMEM are
// released.
#pragma once

#include "common.cuh"

namespace zb {

struct WaitCtl {
    volatile int* abort_flag;  // shared memory, one per CTA
    int* status;               // per-call status word (workspace)
    int* report;               // per-device report word
    unsigned long long limit_ns;
    uint32_t peer_flag = 0;    // CTA pair: shared::cluster address of the other CTA's abort flag
};

ZB_DEVICE void st_cluster_u32(uint32_t cluster_addr, uint32_t v) {
    asm volatile("st.shared::cluster.u32 [%0], %1;\n" ::"r"(cluster_addr), "r"(v) : "memory");
}

// Abort sites recorded in the status / report words.
enum : int {
    WAIT_PRODUCER_EMPTY_A = 1,
    WAIT_PRODUCER_EMPTY_B = 2,
    WAIT_MMA_TEMPTY = 3,
    WAIT_MMA_FULL_A = 4,
    WAIT_MMA_FULL_B = 5,
    WAIT_EPILOGUE_TFULL = 6,
    WAIT_MMA_HOLD = 7,  // test-only hold: a barrier nothing arrives on
};

ZB_DEVICE unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar`; false if another role aborted or the wait
// ran out (then the abort is raised and recorded unless `where` is 0).  The
// poll count is capped as well, in case the timer does not advance.
ZB_DEVICE bool wait_phase(uint64_t* bar, uint32_t parity, const WaitCtl& w, int where) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (uint32_t i = 1; i < (1u << 30); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 0) {
            if (*w.abort_flag) return false;
            if (globaltimer_ns() - t0 > w.limit_ns) break;
        }
    }
    *w.abort_flag = 1;
    if (w.peer_flag) st_cluster_u32(w.peer_flag, 1u);
    if (where) {
        if (w.status) atomicCAS(w.status, 0, where);
        if (w.report) atomicCAS(w.report, 0, where);
    }
    return false;
}

// Abort path: wait (bounded, regardless of the abort flag) for a phase that
// only asynchronous hardware completes (TMA bytes landing, an MMA commit).
ZB_DEVICE bool drain_phase(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
    const unsigned long long t0 = globaltimer_ns();
    for (uint32_t i = 0; i < (1u << 30); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 255 && globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// Spin for `ns` nanoseconds (bounded by a poll count).
ZB_DEVICE void spin_ns(unsigned long long ns) {
    const unsigned long long t0 = globaltimer_ns();
    for (uint32_t i = 0; i < (1u << 24) && globaltimer_ns() - t0 < ns; ++i) __nanosleep(256);
}

// TMA loads issued by the producer and not yet seen consumed: bit s of
// `pending` set when slot s was loaded, bit s of `phase` its ring phase then.
struct Issued {
    uint32_t pending = 0, phase = 0;
    ZB_DEVICE void note(int slot, uint32_t ph) {
        pending |= 1u << slot;
        phase = (phase & ~(1u << slot)) | (ph << slot);
    }
    // Wait for every noted load's bytes (its "full" barrier phase).
    ZB_DEVICE void drain(uint64_t* full, int slots, unsigned long long limit_ns) const {
        for (int s = 0; s < slots; ++s)
            if ((pending >> s) & 1u) drain_phase(&full[s], (phase >> s) & 1u, limit_ns);
    }
};


}  // namespace zb
