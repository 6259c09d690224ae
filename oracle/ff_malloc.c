/* Test infrastructure: the allocator the BFS-like oracle build of the
 * reference's src/sptensor/renumber.c is compiled with (-Dmalloc=pti_ff_malloc,
 * see oracle/Makefile).  ptiBFSLike (renumber.c:794-839) reads the markers of
 * other modes' vertices (renumber.c:768; the same loop in orderit.c:1070)
 * without ever setting them, so its result depends on whatever the allocator
 * returns.  Filling every fresh block with 0xFF bytes makes those markers -1,
 * i.e. "not visited", the reading under which the algorithm is the
 * maximum-cardinality search its comments describe, and makes the result
 * deterministic. */
#include <stdlib.h>
#include <string.h>

void *pti_ff_malloc(size_t n)
{
    void *p = malloc(n);
    if (p) memset(p, 0xff, n);
    return p;
}
