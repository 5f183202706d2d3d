/* The reference installs its ncbi_blast_files/gpu_cpu_common.h into the NCBI
 * tree as algo/blast/core/gpu_cpu_common.h; this forwards that include path
 * to the reference's own file (found through -I<reference root>), so the
 * record layout and ring size are the reference's.  TEST INFRASTRUCTURE ONLY. */
#include <ncbi_blast_files/gpu_cpu_common.h>
