/*
 * Stand-in for NCBI BLAST+ 2.2.28's algo/blast/core/blast_aalookup.h (and
 * the ncbi_std.h / blast_lookup.h names it brings in), holding only what the
 * reference's kernel source and ncbi_blast_files/gpu_cpu_common.h use.
 * TEST INFRASTRUCTURE ONLY: used to host-compile the reference kernel.
 *
 * AaLookupSmallboneCell follows NCBI's published layout (a count, then either
 * AA_HITS_PER_CELL inline 16-bit query offsets or a cursor into the overflow
 * array); PV_TEST is NCBI's presence-vector bit test over an array of 32-bit
 * words.  The NCBI structures that only appear in prototypes stay incomplete.
 */
#ifndef BLASTP_REFSHIM_BLAST_AALOOKUP_H
#define BLASTP_REFSHIM_BLAST_AALOOKUP_H

#include <stdint.h>

typedef int32_t Int4;
typedef uint32_t Uint4;
typedef uint16_t Uint2;
typedef uint8_t Uint1;
typedef uint8_t Boolean;

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif
#ifndef MIN
#define MIN(a, b) ((a) > (b) ? (b) : (a))
#endif
#ifndef MAX
#define MAX(a, b) ((a) >= (b) ? (a) : (b))
#endif

#define PV_ARRAY_TYPE Uint4
#define PV_ARRAY_BTS 5
#define PV_ARRAY_MASK 31
#define PV_TEST(pv, index, shift) \
    ((pv)[(index) >> (shift)] & (((PV_ARRAY_TYPE)1) << ((index) & PV_ARRAY_MASK)))

#define REFSHIM_AA_HITS_PER_CELL 3
typedef struct AaLookupSmallboneCell {
    Int4 num_used;
    union {
        Uint2 entries[REFSHIM_AA_HITS_PER_CELL];
        Int4 overflow_cursor;
    } payload;
} AaLookupSmallboneCell;

typedef struct BLAST_SequenceBlk BLAST_SequenceBlk;
typedef struct BlastQueryInfo BlastQueryInfo;
typedef struct LookupTableWrap LookupTableWrap;
typedef struct Blast_ExtendWord Blast_ExtendWord;
typedef struct BlastInitialWordParameters BlastInitialWordParameters;
typedef struct BlastGPUOptions BlastGPUOptions;

#endif
