// vox_internal.h - interfaces between the CUDA translation units of the
// Gaussian -> node2 library.  Not part of the public C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vox
{

// number of kernels this library has launched (all contexts, all threads)
int64_t launch_count();
void count_launch();

// Bump allocator over one device arena; grows (re-allocates) between calls only.
struct Arena
{
    char* base = nullptr;
    size_t cap = 0;
    size_t used = 0;
    void reset()
    {
        used = 0;
    }
    template <class T>
    T* take(size_t count, size_t align = 256)
    {
        size_t off = (used + align - 1) / align * align;
        size_t bytes = count * sizeof(T);
        if (off + bytes > cap)
            return nullptr;
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

// Look-back bookkeeping: each user owns a status region and an epoch counter
// so that regions need no clearing between uses (epoch wraps every 255 uses,
// at which point the region is cleared once).
struct Epochs
{
    // A region seen for the first time (new allocation) or after 255 uses is
    // cleared once; otherwise stale words carry an older epoch and are ignored.
    uint32_t next(uint64_t* region, size_t words, cudaStream_t s)
    {
        if (value == 255 || value == 0 || region != last_region || words != last_words)
        {
            cudaMemsetAsync(region, 0, words * sizeof(uint64_t), s);
            value = 0;
            last_region = region;
            last_words = words;
        }
        return ++value;
    }
    uint32_t value = 0;
    uint64_t* last_region = nullptr;
    size_t last_words = 0;
};

// ---------------------------------------------------------------- scan ----
// scan of n u64 values; mode bit 0: scan popcounts of the words instead of the
// values, bit 1: inclusive instead of exclusive.  out may alias in; *total
// receives the sum.
size_t scan_status_words(int64_t n);
void scan_exclusive_u64(const uint64_t* in, uint64_t* out, int64_t n, int mode, uint64_t* total, uint64_t* status,
                        uint32_t epoch, uint32_t* counter, int* err, int num_sms, cudaStream_t s);

// u32 scan (sum mod 2^32, or running maximum with max_op), inclusive or
// exclusive; *total (u64) receives the sum / maximum
void scan_u32(const uint32_t* in, uint32_t* out, int64_t n, int inclusive, int max_op, uint64_t* total,
              uint64_t* status, uint32_t epoch, uint32_t* counter, int* err, cudaStream_t s);
// dual-key sort helpers: key = (high & mask) << low_bits | (low & mask), idx = i;
// then low / high / val gathered through the sorted idx from copies
void dual_combine(const uint32_t* low, const uint32_t* high, int64_t n, int low_bits, int high_bits, uint64_t* key,
                  uint32_t* idx, int num_sms, cudaStream_t s);
void dual_gather(const uint32_t* sidx, int64_t n, const uint32_t* low_c, const uint32_t* high_c, const uint32_t* val_c,
                 uint32_t* low, uint32_t* high, uint32_t* val, int* err, int num_sms, cudaStream_t s);

// Online choice among launch variants that give identical results.  Per size
// class (floor(log2) of the work), the first call of a class is a warm-up
// (its time, taken on freshly mapped buffers, is not used), then each call of
// a class that has untried variants runs the next one and reports its time per
// unit of work; later calls run the fastest.  No extra work is launched to tune.
struct OnlineChoice
{
    static const int kClasses = 40, kMax = 4;
    int variants = 1;
    float cost[kClasses][kMax];
    bool warm[kClasses];
    explicit OnlineChoice(int n = 1) : variants(n)
    {
        for (auto& r : cost)
            for (float& c : r)
                c = -1.f;
        for (bool& w : warm)
            w = false;
    }
    static int size_class(int64_t work)
    {
        int c = 0;
        while (c < kClasses - 1 && (1ll << (c + 1)) <= work)
            c++;
        return c;
    }
    int pick(int64_t work) const
    {
        const int c = size_class(work);
        int best = 0;
        for (int v = 0; v < variants; v++)
        {
            if (cost[c][v] < 0.f)
                return v;
            if (cost[c][v] < cost[c][best])
                best = v;
        }
        return best;
    }
    void report(int64_t work, int v, float ms)
    {
        const int c = size_class(work);
        if (!warm[c])
        {
            warm[c] = true;
            return;
        }
        if (v >= 0 && v < variants && work > 0 && cost[c][v] < 0.f && ms > 0.f)
            cost[c][v] = ms / (float)work;
    }
};

// ---------------------------------------------------------------- sort ----
struct SortTuning
{
    int digit_bits = 8; // radix bits per pass (<= 8)
    int shape = -1;     // onesweep tile shape, -1 = tuned: fastest pass 0 per key width and size class
    int best[2][40];    // tuner's choice per (64-bit keys, floor(log2 n)), -1 = not yet timed
    SortTuning()
    {
        for (auto& r : best)
            for (int& b : r)
                b = -1;
    }
};
size_t sort_workspace_bytes(int64_t n, int key_bytes);
// Stable LSD sort of (key, value) pairs by key bits [0, key_bits) (higher
// bits take no part in the order).  Uses
// keys_alt / vals_alt as ping-pong buffers; returns 0 if the result is in
// keys / vals and 1 if it is in keys_alt / vals_alt.
int sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                   void* workspace, Epochs* epochs, int* err, int num_sms, cudaStream_t s, SortTuning& tune);
int sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                   void* workspace, Epochs* epochs, int* err, int num_sms, cudaStream_t s, SortTuning& tune);
size_t sort_status_words(int64_t n);
// shape index the sort of n pairs uses under `tune` (-1 before tuning)
int sort_shape_used(int64_t n, int key64, const SortTuning& tune);

// counts keys[i] < keys[i - 1] into *descents (validation)
void check_sorted(const void* keys, int64_t n, int key64, uint64_t* descents, int num_sms, cudaStream_t s);

} // namespace vox
