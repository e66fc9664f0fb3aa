// hostcopy.h -- the host copy pool behind the non-zero-copy paths.
//
// Callers that hand the decoder ordinary (pageable) host buffers pay one host
// memcpy per byte: inputs into a page-locked staging buffer before their DMA,
// outputs from a page-locked buffer into the caller's memory after theirs.
// One thread copies at a few GB/s, slower than the PCIe DMA and often slower
// than the decode itself; the pool spreads every copy over several threads
// (the calling thread included) in 1 MiB pieces.
//
// Threads: HPVCD_COPY_THREADS when set (0 = copy on the calling thread only),
// else half the hardware threads, at most 8.  They are started on first use
// and live for the rest of the process.
#pragma once

#include <stddef.h>

namespace hpvcd_host {

struct CopyTask {
    void* dst;
    const void* src;
    size_t bytes;
};

// Copy every task (dst and src ranges must not overlap); returns when all
// bytes have landed.  Safe to call from several threads at once.
void parallel_copy(const CopyTask* tasks, size_t n);

inline void parallel_copy(void* dst, const void* src, size_t bytes) {
    const CopyTask t{dst, src, bytes};
    parallel_copy(&t, 1);
}

// Worker threads of the pool (not counting callers).
int copy_threads();

}  // namespace hpvcd_host
