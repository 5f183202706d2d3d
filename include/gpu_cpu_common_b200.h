/*
 * gpu_cpu_common_b200.h -- the reference's GPU entry points, served by the
 * B200 engine.  A drop-in for the plain single-query GPU call that NCBI's
 * preliminary search makes (ncbi_blast_files/functions.cpp:641-699,
 * 1099,1328,1407; blast_engine.c:1575), with the reference's names,
 * parameter lists, buffer layouts and ownership rules.
 *
 * Entry point                    replaces (file:line in the reference)
 *   GPU_BLASTP                     gpu_blastp.cu:16-222, gpu_cpu_common.h:44-63
 *   GPU_BLASTP_get_data            gpu_blastp.cu:224-259, gpu_cpu_common.h:65-69
 *   GPU_BLASTP_free_memory         gpu_blastp.cu:262-280, gpu_cpu_common.h:71-79
 *   GPU_BLASTP_check_memory        gpu_blastp.cu:282-334, gpu_cpu_common.h:81-89
 *   GPU_BLAST_check_availability   gpu_blastp.cu:336-344, gpu_cpu_common.h:91
 *   Round2Multiple                 gpu_blastp.c:12-17,    gpu_cpu_common.h:93
 *
 * Contract kept: the caller owns the nine device-pointer slots (NULL on
 * entry), GPU_BLASTP fills them and returns once the search is enqueued (its
 * host-to-device copies are synchronous, so the caller may free the host
 * database right away); GPU_BLASTP_get_data is the synchronisation point and
 * copies d_Hits[oid*3+{hits, successful extensions, extensions}] and the
 * two-slot-per-subject HSP ring to the host; GPU_BLASTP_free_memory frees the
 * slots.  What changed behind it: the slots hold this engine's buffers, every
 * CUDA call is checked, and the ring is filled from the complete, ordered HSP
 * set.  On a failure the cause is printed and every subject's counters read
 * {0 hits, 3 successful extensions, 0 extensions}: more successful
 * extensions than the two ring slots hold, which is the condition under
 * which NCBI's ingestion re-searches a subject on the CPU
 * (blast_engine.c:529-538), so no subject is silently dropped.
 *
 * Build inside the NCBI tree with -DBLASTP_B200_WITH_NCBI so the NCBI types
 * come from NCBI's headers; otherwise they come from ncbi_compat.h.
 */
#ifndef GPU_CPU_COMMON_B200_H
#define GPU_CPU_COMMON_B200_H

#ifdef BLASTP_B200_WITH_NCBI
#include <algo/blast/core/blast_aalookup.h>
#include <algo/blast/core/blast_extend.h>
#include <algo/blast/core/blast_options.h>
#include <algo/blast/core/lookup_wrap.h>
#else
#include "ncbi_compat.h"
#endif

#define MAX_SUCCESSFUL_HITS_PER_SEQUENCE 2   /* gpu_cpu_common.h:11 */
#define QUERY_LENGTH_MAX_B200 65535          /* reference: 16384 (gpu_cpu_common.h:25) */
#define NUM_QUERIES_MAX_B200 65536           /* reference: 4096 (gpu_cpu_common.h:26) */

#ifndef GPU_CPU_COMMON_H
typedef struct GPUBlastInitHitList {          /* gpu_cpu_common.h:29-38 */
    int hsp_q;
    int hsp_s;
    int query_offset;
    int subject_offset;
    int hsp_len;
    int score;
} GPUBlastInitHitList;
#endif

#ifdef __cplusplus
extern "C" {
#endif

void GPU_BLASTP(const BLAST_SequenceBlk* query, const BlastQueryInfo* query_info,
                const LookupTableWrap* lookup_wrap, const Blast_ExtendWord* ewp,
                const BlastInitialWordParameters* word_params, const BlastGPUOptions* gpu_options,
                const int* Sequence_length_vector, const int h_Database2Dpadded_bytes,
                const char* h_Database2Dpadded, Int4** d_Hits, const Int4 h_Hits_bytes,
                GPUBlastInitHitList** d_GPUBlastInitHitList, const Int4 h_GPUBlastInitHitList_bytes,
                Int4** d_Database2Dpadded, Int4** d_RepeatedSubstitutionMatrix,
                Int4** d_RepeatedSequence_length_vector, PV_ARRAY_TYPE** d_RepeatedPV,
                AaLookupSmallboneCell** d_ThickBackbone, Uint2** d_overflow,
                Int4** d_RepeatedDiag_array);

void GPU_BLASTP_get_data(Int4* h_Hits, Int4* d_Hits, const Int4 h_Hits_bytes,
                         GPUBlastInitHitList* h_GPUBlastInitHitList,
                         GPUBlastInitHitList* d_GPUBlastInitHitList, Int4 h_GPUBlastInitHitList_bytes,
                         Int4 num_sequences);

void GPU_BLASTP_free_memory(Int4** d_Hits, GPUBlastInitHitList** d_GPUBlastInitHitList,
                            Int4** d_Database2Dpadded, Int4** d_RepeatedSubstitutionMatrix,
                            Int4** d_RepeatedSequence_length_vector, PV_ARRAY_TYPE** d_RepeatedPV,
                            AaLookupSmallboneCell** d_ThickBackbone, Uint2** d_overflow,
                            Int4** d_RepeatedDiag_array);

Boolean GPU_BLASTP_check_memory(const LookupTableWrap* lookup_wrap, const Blast_ExtendWord* ewp,
                                const BlastGPUOptions* gpu_options, const int h_Database2Dpadded_bytes,
                                const Int4 h_Hits_bytes, const Int4 h_GPUBlastInitHitList_bytes,
                                const Int4 Group_number, const Int4 num_queries, const Int4 query_length);

Boolean GPU_BLAST_check_availability(void);

void Round2Multiple(Int4* MaxLength);

/* Addition (no counterpart in the reference): the complete HSP set of the
 * last GPU_BLASTP call on d_Hits, valid between GPU_BLASTP_get_data and
 * GPU_BLASTP_free_memory.  hsp_off[num_sequences+1] (int64) indexes hsps per
 * subject, in discovery order.  With it a caller fills its initial-hit lists
 * for every subject, including those with more than two HSPs, which the
 * two-slot ring cannot hold and which the reference sends back to the CPU
 * (blast_engine.c:529-538).  hsps may be NULL to learn the count (n_hsps);
 * returns FALSE when there is no such search, it failed, or hsp_cap is too
 * small. */
Boolean GPU_BLASTP_get_hsps(Int4* d_Hits, int64_t* hsp_off, GPUBlastInitHitList* hsps, int64_t hsp_cap,
                            int64_t* n_hsps);

#ifdef __cplusplus
}
#endif

#endif /* GPU_CPU_COMMON_B200_H */
