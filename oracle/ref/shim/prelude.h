/* prelude.h -- force-included when compiling the reference's C sources with
 * gcc (oracle/ref/Makefile).  Test infrastructure only.
 * Stands in for Intel-compiler features the sources use:
 *   __declspec(align(64))   pscf/purif.h:66, pscf/purif.c:613-614
 *   _castf64_u64            pfock/fock_task.c:22-23
 *   _mm_malloc/_mm_free     pfock/config.h:13-14 (zero-filled here, so the
 *                           fields PFock_create leaves unset read as zero)
 */
#ifndef GTF_REF_PRELUDE_H
#define GTF_REF_PRELUDE_H
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#define __declspec(x)
static inline uint64_t _castf64_u64(double d)
{
    uint64_t u;
    memcpy(&u, &d, sizeof(u));
    return u;
}
void *gtf_ref_aligned_calloc(size_t size, size_t align);
#define _mm_malloc(size, align) gtf_ref_aligned_calloc((size), (align))
#define _mm_free(p) free(p)
#endif
