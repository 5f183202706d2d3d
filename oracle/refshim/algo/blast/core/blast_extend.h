/* Stand-in for NCBI BLAST+ 2.2.28's algo/blast/core/blast_extend.h: nothing from it is
 * used by the reference kernel; the names the reference's gpu_cpu_common.h
 * needs come from blast_aalookup.h.  TEST INFRASTRUCTURE ONLY. */
#include <algo/blast/core/blast_aalookup.h>
