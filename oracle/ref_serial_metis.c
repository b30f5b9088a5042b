/* Serial stand-ins for the three graph-partitioning entry points that the
 * reference's mesh set-up calls even for a single process
 * (meshPreProcess/decomposing/src/decomposingByMetis.cpp:111-137). With one
 * part every cell belongs to part 0, which is what a real partitioner returns
 * for nparts == 1; any other part count is refused. Test infrastructure for
 * the oracle driver only (linked into oracle/_ref/hurchem_ref). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef int32_t idx_t;
typedef float real_t;

int METIS_SetDefaultOptions(idx_t *options) {
    for (int i = 0; i < 40; ++i) options[i] = -1;
    return 1;
}

static int one_part(idx_t *nvtxs, idx_t *nparts, idx_t *edgecut, idx_t *part) {
    if (*nparts != 1) {
        fprintf(stderr, "serial partition stand-in asked for %d parts\n", (int)*nparts);
        abort();
    }
    for (idx_t i = 0; i < *nvtxs; ++i) part[i] = 0;
    if (edgecut) *edgecut = 0;
    return 1;
}

int METIS_PartGraphRecursive(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy, idx_t *vwgt,
                             idx_t *vsize, idx_t *adjwgt, idx_t *nparts, real_t *tpwgts,
                             real_t *ubvec, idx_t *options, idx_t *edgecut, idx_t *part) {
    (void)ncon; (void)xadj; (void)adjncy; (void)vwgt; (void)vsize; (void)adjwgt;
    (void)tpwgts; (void)ubvec; (void)options;
    return one_part(nvtxs, nparts, edgecut, part);
}

int METIS_PartGraphKway(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy, idx_t *vwgt,
                        idx_t *vsize, idx_t *adjwgt, idx_t *nparts, real_t *tpwgts,
                        real_t *ubvec, idx_t *options, idx_t *edgecut, idx_t *part) {
    (void)ncon; (void)xadj; (void)adjncy; (void)vwgt; (void)vsize; (void)adjwgt;
    (void)tpwgts; (void)ubvec; (void)options;
    return one_part(nvtxs, nparts, edgecut, part);
}
