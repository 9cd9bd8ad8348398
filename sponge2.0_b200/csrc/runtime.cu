// Error reporting, stream selection and small host utilities of the C ABI.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <stdlib.h>

#include "common.cuh"

namespace spgnb
{
namespace
{
thread_local char g_last_error[1024] = "";
thread_local cudaStream_t g_stream = nullptr;
thread_local cudaEvent_t g_pair_start = nullptr, g_pair_stop = nullptr;
unsigned long long g_launches = 0;
}  // namespace

void count_launch() { __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED); }
void count_launches(long long n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }
unsigned long long launches_so_far() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

// SPGNB_SYNC_CHECK=1: every launch is followed by a device synchronisation so
// that an execution error is reported against the kernel that caused it.
bool sync_check()
{
    static const bool on = [] {
        const char* v = getenv("SPGNB_SYNC_CHECK");
        return v && v[0] == '1';
    }();
    return on;
}

void pair_events(cudaEvent_t* start, cudaEvent_t* stop)
{
    *start = g_pair_start;
    *stop = g_pair_stop;
}

unsigned long long launches() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
void set_pair_events(cudaEvent_t a, cudaEvent_t b)
{
    g_pair_start = a;
    g_pair_stop = b;
}

int fail(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(SPGNB_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

cudaStream_t stream() { return g_stream; }

int num_sms()
{
    static int cached = 0;
    if (cached == 0)
    {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cached = v;
    }
    return cached;
}

}  // namespace spgnb

extern "C" {

const char* spgnb_version(void) { return "spgnb 0.1 (sm_100a)"; }

const char* spgnb_status_string(int status)
{
    switch (status)
    {
        case SPGNB_OK:
            return "ok";
        case SPGNB_E_ARG:
            return "invalid argument";
        case SPGNB_E_OOM:
            return "device allocation failed";
        case SPGNB_E_CUDA:
            return "CUDA error";
        case SPGNB_E_OVERFLOW:
            return "buffer overflow";
        case SPGNB_E_NONFINITE:
            return "non-finite result";
        case SPGNB_E_STATE:
            return "call out of order";
        case SPGNB_E_TIMEOUT:
            return "device wait timed out";
        case SPGNB_E_UNSUPPORTED:
            return "unsupported configuration";
        default:
            return "unknown status";
    }
}

const char* spgnb_last_error(void) { return spgnb::g_last_error; }

unsigned long long spgnb_launch_count(void) { return spgnb::launches(); }

int spgnb_debug_set_pair_events(void* start_event, void* stop_event)
{
    spgnb::set_pair_events((cudaEvent_t)start_event, (cudaEvent_t)stop_event);
    return SPGNB_OK;
}

int spgnb_set_stream(void* cuda_stream)
{
    spgnb::g_stream = (cudaStream_t)cuda_stream;
    return SPGNB_OK;
}

// Ewald splitting parameter for a direct-space cutoff: the beta at which the
// screened Coulomb kernel erfc(beta rc)/rc falls to `tolerance`.  The search
// is the one SPONGE runs (PM_force.cpp:244-272), so the value is bit-identical
// to the reference's: an upper bound doubled from 1 until the kernel is at or
// below the tolerance, then (doublings + 50) halvings of [0, bound], each
// keeping the half where the kernel is still >= the tolerance; the answer is
// the last midpoint, all in float.
float spgnb_get_beta(float cutoff, float tolerance)
{
    if (!(cutoff > 0.0f) || !(tolerance > 0.0f)) return 0.0f;
    const auto screened = [cutoff](float b) { return erfcf(b * cutoff) / cutoff; };
    float hi = 1.0f;
    int doublings = 0;
    while (screened(hi) > tolerance)
    {
        hi *= 2.0f;
        ++doublings;
    }
    float lo = 0.0f, mid = 0.0f;
    for (int step = 0; step < doublings + 50; ++step)
    {
        mid = 0.5f * (lo + hi);
        if (screened(mid) >= tolerance)
            lo = mid;
        else
            hi = mid;
    }
    return mid;
}

}  // extern "C"
