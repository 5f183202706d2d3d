/*
 * ncbi_compat.h -- stand-ins for the NCBI BLAST+ 2.2.28 types that the
 * GPU_BLASTP entry points take, for builds outside the NCBI tree.
 *
 * The reference declares its entry points over NCBI's own structures
 * (ncbi_blast_files/gpu_cpu_common.h:6-9,44-93) and reads a handful of their
 * fields (gpu_blastp.cu:26-82, 208-209).  Inside an NCBI build this library's
 * shim is compiled with -DBLASTP_B200_WITH_NCBI against NCBI's real headers,
 * so the layouts are NCBI's.  Outside it (this repository's tests), the
 * structures below stand in: each carries exactly the fields the shim reads,
 * under NCBI's field names, in an order of this file's own choosing.  They are
 * NOT layout-compatible with NCBI's structures and must not be mixed with
 * objects built by NCBI code.
 *
 * BlastGPUOptions and GPUBlastInitHitList are the reference's own types
 * (ncbi_blast_files/blast_options.h:484-494, gpu_cpu_common.h:29-38) and are
 * reproduced with their layouts.
 */
#ifndef BLASTP_B200_NCBI_COMPAT_H
#define BLASTP_B200_NCBI_COMPAT_H

#include <stdint.h>

typedef int32_t Int4;
typedef uint32_t Uint4;
typedef uint16_t Uint2;
typedef uint8_t Uint1;
typedef uint8_t Boolean;
typedef unsigned int PV_ARRAY_TYPE;   /* gpu_blastp.h:8 */

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

#define PV_ARRAY_BTS 5                /* log2 of the bits in a PV_ARRAY_TYPE */
#define AA_HITS_PER_CELL 3            /* inline query offsets per backbone cell */

typedef struct BLAST_SequenceBlk {
    Uint1* sequence;                  /* concatenated query contexts */
    Int4 length;
} BLAST_SequenceBlk;

typedef struct BlastContextInfo {
    Int4 query_offset;                /* first residue of the context */
} BlastContextInfo;

typedef struct BlastQueryInfo {
    Int4 num_queries;
    BlastContextInfo* contexts;
} BlastQueryInfo;

typedef struct AaLookupSmallboneCell {
    Int4 num_used;                    /* query offsets listed under this word */
    union {
        Uint2 entries[AA_HITS_PER_CELL];   /* when num_used <= 3 */
        Int4 overflow_cursor;              /* else: start in the overflow array */
    } payload;
} AaLookupSmallboneCell;

typedef struct BlastAaLookupTable {
    Int4 mask;                        /* index mask, 2^(word*charsize) - 1 */
    Int4 charsize;                    /* bits per letter */
    Int4 word_length;
    Int4 backbone_size;               /* cells in thick_backbone */
    void* thick_backbone;             /* AaLookupSmallboneCell[backbone_size] */
    void* overflow;                   /* Uint2[overflow_size] */
    Int4 overflow_size;
    PV_ARRAY_TYPE* pv;                /* presence bits, one per cell */
} BlastAaLookupTable;

typedef struct LookupTableWrap {
    Int4 lut_type;
    void* lut;                        /* BlastAaLookupTable* for blastp */
} LookupTableWrap;

typedef struct BLAST_DiagTable {
    Int4 diag_array_length;           /* power of two >= query length + window */
    Int4 diag_mask;                   /* diag_array_length - 1 */
    Int4 offset;                      /* running diagonal offset, starts at window */
    Int4 window;                      /* two-hit window */
} BLAST_DiagTable;

typedef struct Blast_ExtendWord {
    BLAST_DiagTable* diag_table;
} Blast_ExtendWord;

typedef struct BlastUngappedCutoffs {
    Int4 x_dropoff;                   /* raw X-drop for this context */
    Int4 cutoff_score;                /* raw score to report an HSP */
} BlastUngappedCutoffs;

typedef struct BlastInitialWordParameters {
    BlastUngappedCutoffs* cutoffs;    /* one per context */
} BlastInitialWordParameters;

typedef struct BlastGPUOptions {      /* blast_options.h:484-494 */
    char use_gpu;
    int num_blocksx;
    int num_threadsx;
    int num_sequences_to;
    int method;
    int cpu_threads;
} BlastGPUOptions;

#endif /* BLASTP_B200_NCBI_COMPAT_H */
