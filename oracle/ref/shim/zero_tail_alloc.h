// Allocator for kipl image buffers in the reference oracle (test infrastructure only).
//
// kipl::base::buffer allocates its images with _mm_malloc((N + 16) * sizeof(T), 32)
// (core/kipl/kipl/include/base/core/sharedbuffer.h:66-75) and leaves the memory
// uninitialised. The reference's median filter (TMedianFilter::ExtractNeighborhood) reads a
// few values past the end of the image near its bottom-right corner, so its result there
// depends on whatever the heap held. Force-included into every translation unit of the
// oracle, this header routes those allocations to a block with 1 MiB of slack behind it and
// zeroes the block's last 256 bytes (which cover the 16-element tail for every element type
// kipl uses, at most 16 bytes each) and the slack: the out-of-image reads then return 0, the
// value the restatement and the CUDA path use there. The image data itself is left as the
// reference leaves it (so the timed reference runs pay no extra pass), and nothing else about
// the reference changes.
#ifndef ORACLE_ZERO_TAIL_ALLOC_H
#define ORACLE_ZERO_TAIL_ALLOC_H

#include <mm_malloc.h>
#include <stdlib.h>
#include <string.h>

static inline void *oracle_zero_tail_malloc(size_t size, size_t align)
{
    const size_t slack = size_t(1) << 20;
    void *p = 0;
    if (align < sizeof(void *)) align = sizeof(void *);
    if (posix_memalign(&p, align, size + slack) != 0) return 0;
    const size_t tail = size < 256 ? size : 256;
    memset(static_cast<char *>(p) + (size - tail), 0, tail + slack);
    return p;
}

#define _mm_malloc(size, align) oracle_zero_tail_malloc((size), (align))

#endif
