// Host side of the C ABI's bulk copies: a pool of host worker threads and
// pinned staging chunks between pageable user buffers and device planes.
//
// The reference copies its host arrays with plain synchronous cudaMemcpy from
// pageable memory (GPU/main_TSUNER.cu:113-122 upload, :159-162 and :199-207
// read-back).  A pageable copy runs through one driver thread at a fraction of
// the link rate, and a read-back into memory the process has not touched yet
// also pays one page fault per 4 KB page on that thread.  Here the DMA engine
// only reads/writes pinned chunks, at link rate, while the pool moves bytes
// between those chunks and the user's buffer (faulting its pages in parallel)
// for the previous chunk.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <functional>

namespace tsu {

// Worker threads of the pool (TSU_HOST_THREADS, default min(cores, 16)).
int host_threads();

// fn(i) for every i in [0, n), spread over the pool; the caller takes part and
// returns when all n calls have returned.  Calls from several threads are
// serialised; fn must not call host_parallel itself.
void host_parallel(int n, const std::function<void(int)> &fn);

// Fills `nr` rows of plane `plane`, starting at row `r0`, into `dst` (rows of
// `width` bytes back to back); used when the host layout is not the device
// layout (e.g. an int mask stored as bytes).  Called in parallel on disjoint
// row ranges.
using RowFill = std::function<void(int plane, size_t r0, size_t nr, unsigned char *dst)>;

// `nplanes` planes of `rows` rows x `width` bytes: host plane p at host[p]
// with row pitch `hpitch`, device plane p at dev[p] with row pitch `dpitch`.
// Ordered on `st` after the work already queued there; both return when the
// copy has completed (the stream is synchronised).  `fill`, when given,
// replaces the plain row copy from host[p].
cudaError_t planes_h2d(int nplanes, void *const *dev, size_t dpitch, const void *const *host, size_t hpitch,
                       size_t width, size_t rows, cudaStream_t st, const RowFill &fill = RowFill());
cudaError_t planes_d2h(int nplanes, void *const *host, size_t hpitch, const void *const *dev, size_t dpitch,
                       size_t width, size_t rows, cudaStream_t st);

// Contiguous byte ranges.
cudaError_t bytes_h2d(void *dev, const void *host, size_t bytes, cudaStream_t st);
cudaError_t bytes_d2h(void *host, const void *dev, size_t bytes, cudaStream_t st);

}  // namespace tsu
