// Process-global structured trace ring (4096 x 64-byte events, drop-oldest)
// and the POSIX crash dump that snapshots it on SIGSEGV/SIGABRT/SIGFPE/SIGBUS.
//
// Reference semantics followed (project-relative paths):
//   ring        L1-native/libpfsf/src/trace/ring_buffer.cpp:20-201
//   crash dump  L1-native/libpfsf/src/diag/crash.cpp:40-301
//
// Dump file format (shared with the reference so its readers keep working):
//   "PFSF-CRASH signo=<dec> pid=<dec> addr=0x<lowercase hex> events=<dec>\n"
//   followed by <events> raw pfsf_trace_event records, oldest first, at most
//   PFSF_CRASH_MAX_EVENTS of the newest.
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <fcntl.h>
#include <signal.h>
#include <unistd.h>

#include "pfsf/pfsf_trace.h"

namespace {

static_assert(sizeof(pfsf_trace_event) == 64, "trace events are a frozen 64-byte wire format");
constexpr uint32_t kRing = PFSF_TRACE_RING_CAPACITY;

// Namespace-scope, constant-initialised state: the signal handler may read
// it before any emit ever ran, so there must be no first-use guard.
struct Ring {
    std::mutex mu;
    pfsf_trace_event ev[kRing];
    uint32_t head;   // next slot to write
    uint32_t count;  // live events (<= kRing)
};
Ring g_ring{};
std::atomic<int32_t> g_level{PFSF_TRACE_INFO};

// Copies the newest min(cap, live) events, oldest of them first, without the
// lock (best effort: used from the signal handler).
int32_t peek_newest(pfsf_trace_event* out, int32_t cap) {
    uint32_t live = g_ring.count, head = g_ring.head;
    if (live > kRing) live = kRing;
    const uint32_t n = cap < int32_t(live) ? uint32_t(cap) : live;
    for (uint32_t i = 0; i < n; ++i) out[i] = g_ring.ev[(head + kRing - n + i) % kRing];
    return int32_t(n);
}

// Async-signal-safe formatting: decimal / lowercase hex into buf.
int put_dec(int64_t v, char* buf) {
    char t[24];
    int n = 0;
    uint64_t u = v < 0 ? uint64_t(-(v + 1)) + 1u : uint64_t(v);
    do {
        t[n++] = char('0' + u % 10);
        u /= 10;
    } while (u);
    int k = 0;
    if (v < 0) buf[k++] = '-';
    while (n) buf[k++] = t[--n];
    return k;
}

int put_hex(uintptr_t v, char* buf) {
    char t[24];
    int n = 0;
    do {
        const unsigned d = unsigned(v & 15u);
        t[n++] = char(d < 10 ? '0' + d : 'a' + d - 10);
        v >>= 4;
    } while (v);
    int k = 0;
    while (n) buf[k++] = t[--n];
    return k;
}

// Writes the dump; uses only open/write/close/getpid.  Returns the number of
// events written or PFSF_ERROR_VULKAN when the file cannot be opened (the
// reference's generic failure code).
int32_t write_dump(int signo, uintptr_t addr, const char* path) {
    char name[64];
    if (!path) {
        int k = 0;
        for (const char* s = "pfsf-crash-"; *s;) name[k++] = *s++;
        k += put_dec(int64_t(::getpid()), name + k);
        for (const char* s = ".trace"; *s;) name[k++] = *s++;
        name[k] = '\0';
        path = name;
    }
    const int fd = ::open(path, O_CREAT | O_WRONLY | O_TRUNC, 0644);
    if (fd < 0) return PFSF_ERROR_VULKAN;
    pfsf_trace_event ev[PFSF_CRASH_MAX_EVENTS];
    const int32_t got = peek_newest(ev, PFSF_CRASH_MAX_EVENTS);
    char line[160];
    int k = 0;
    auto lit = [&](const char* s) {
        while (*s) line[k++] = *s++;
    };
    lit("PFSF-CRASH signo=");
    k += put_dec(signo, line + k);
    lit(" pid=");
    k += put_dec(int64_t(::getpid()), line + k);
    lit(" addr=0x");
    k += put_hex(addr, line + k);
    lit(" events=");
    k += put_dec(got, line + k);
    line[k++] = '\n';
    ssize_t w = ::write(fd, line, size_t(k));
    if (got > 0) w = ::write(fd, ev, sizeof(pfsf_trace_event) * size_t(got));
    (void)w;
    ::close(fd);
    return got;
}

constexpr int kSignals[] = {SIGSEGV, SIGABRT, SIGFPE, SIGBUS};
constexpr int kNSig = int(sizeof(kSignals) / sizeof(kSignals[0]));
struct sigaction g_prev[kNSig];
volatile sig_atomic_t g_installed = 0;

// Dump, chain to whatever handler was there before (the JVM's hs_err
// writer, a sanitizer), then die with the default action so a returning
// upstream handler cannot swallow the fatal signal.
void on_fatal(int signo, siginfo_t* info, void* ctx) {
    write_dump(signo, info ? uintptr_t(info->si_addr) : 0, nullptr);
    for (int i = 0; i < kNSig; ++i) {
        if (kSignals[i] != signo) continue;
        const struct sigaction& p = g_prev[i];
        if (p.sa_flags & SA_SIGINFO) {
            if (p.sa_sigaction) p.sa_sigaction(signo, info, ctx);
        } else if (p.sa_handler != SIG_DFL && p.sa_handler != SIG_IGN && p.sa_handler) {
            p.sa_handler(signo);
        }
    }
    struct sigaction dfl {};
    dfl.sa_handler = SIG_DFL;
    sigemptyset(&dfl.sa_mask);
    sigaction(signo, &dfl, nullptr);
    raise(signo);
}

}  // namespace

extern "C" {

PFSF_API void pfsf_trace_emit(int16_t level, int64_t epoch, int32_t stage, int32_t island_id, int32_t voxel_index,
                              int32_t errno_val, const char* msg) {
    const int32_t thr = g_level.load(std::memory_order_relaxed);
    if (thr == PFSF_TRACE_OFF || int32_t(level) > thr) return;
    std::lock_guard<std::mutex> lk(g_ring.mu);
    pfsf_trace_event& e = g_ring.ev[g_ring.head];
    e.epoch = epoch;
    e.stage = stage;
    e.island_id = island_id;
    e.voxel_index = voxel_index;
    e.errno_val = errno_val;
    e.level = level;
    e._pad = 0;
    // truncate to 35 bytes + NUL and zero the tail so records are deterministic
    size_t n = 0;
    if (msg)
        while (n < sizeof(e.msg) - 1 && msg[n]) ++n;
    if (n) std::memcpy(e.msg, msg, n);
    std::memset(e.msg + n, 0, sizeof(e.msg) - n);
    g_ring.head = (g_ring.head + 1) % kRing;
    if (g_ring.count < kRing) ++g_ring.count;
}

// Moves up to `capacity` events, oldest first, into out_addr (bounded by
// out_bytes), removing them from the ring.  A NULL buffer is accepted only
// with capacity 0 (and then moves nothing).
PFSF_API int32_t pfsf_drain_trace_dbb(void* out_addr, int64_t out_bytes, int32_t capacity) {
    if (capacity < 0 || (capacity > 0 && !out_addr)) return PFSF_ERROR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_ring.mu);
    int32_t n = int32_t(g_ring.count) < capacity ? int32_t(g_ring.count) : capacity;
    if (out_addr && int64_t(n) * int64_t(sizeof(pfsf_trace_event)) > out_bytes)
        n = int32_t(out_bytes / int64_t(sizeof(pfsf_trace_event)));
    uint32_t at = (g_ring.head + kRing - g_ring.count) % kRing;
    auto* out = static_cast<pfsf_trace_event*>(out_addr);
    for (int32_t i = 0; i < n; ++i, at = (at + 1) % kRing)
        if (out) out[i] = g_ring.ev[at];
    g_ring.count -= uint32_t(n);
    return n;
}

PFSF_API int32_t pfsf_drain_trace(pfsf_engine, pfsf_trace_event* out, int32_t capacity) {
    return pfsf_drain_trace_dbb(out, int64_t(capacity) * int64_t(sizeof(pfsf_trace_event)), capacity);
}

PFSF_API void pfsf_set_trace_level_global(pfsf_trace_level level) { g_level.store(int32_t(level)); }

PFSF_API int32_t pfsf_get_trace_level_global(void) { return g_level.load(); }

PFSF_API void pfsf_set_trace_level(pfsf_engine, pfsf_trace_level level) { pfsf_set_trace_level_global(level); }

PFSF_API int32_t pfsf_trace_size(void) {
    std::lock_guard<std::mutex> lk(g_ring.mu);
    return int32_t(g_ring.count);
}

PFSF_API void pfsf_trace_clear(void) {
    std::lock_guard<std::mutex> lk(g_ring.mu);
    g_ring.head = 0;
    g_ring.count = 0;
}

// Installs the fatal-signal dump (idempotent).  BR_PFSF_NO_SIGNAL set to a
// non-empty value other than "0" skips installation (debuggers, sanitizers).
// An existing handler's SA_ONSTACK is kept so a JVM's alternate-stack
// overflow handling still works when chained.
PFSF_API pfsf_result pfsf_install_crash_handler(void) {
    if (g_installed) return PFSF_OK;
    const char* skip = std::getenv("BR_PFSF_NO_SIGNAL");
    if (skip && skip[0] && skip[0] != '0') return PFSF_OK;
    for (int i = 0; i < kNSig; ++i) {
        struct sigaction cur {};
        if (sigaction(kSignals[i], nullptr, &cur) != 0) cur = {};
        struct sigaction sa {};
        sa.sa_sigaction = on_fatal;
        sa.sa_flags = SA_SIGINFO | SA_RESTART | (cur.sa_flags & SA_ONSTACK);
        sigemptyset(&sa.sa_mask);
        if (sigaction(kSignals[i], &sa, &g_prev[i]) != 0) {
            for (int j = 0; j < i; ++j) sigaction(kSignals[j], &g_prev[j], nullptr);
            return PFSF_ERROR_VULKAN;
        }
    }
    g_installed = 1;
    return PFSF_OK;
}

PFSF_API void pfsf_uninstall_crash_handler(void) {
    if (!g_installed) return;
    for (int i = 0; i < kNSig; ++i) sigaction(kSignals[i], &g_prev[i], nullptr);
    g_installed = 0;
}

// Writes the same file the handler would, synchronously, without a signal.
PFSF_API int32_t pfsf_dump_now_for_test(const char* path, int32_t signo, uintptr_t fault_addr) {
    if (!path) return PFSF_ERROR_INVALID_ARG;
    return write_dump(int(signo), fault_addr, path);
}

}  // extern "C"
