/*
 * A stand-in for WFA2-lib's wavefront/wavefront_align.h, written for this
 * project (WFA2-lib is not available: the reference's WFA2-lib/ submodule
 * is empty, .gitmodules:1-3).  It declares only the names the reference's
 * wfa_gpu.cu uses in its check=1 branch (wfa_gpu.cu:9-11,154-165), so that
 * file compiles unchanged.  The harness never takes that branch: the
 * definitions in ref_stub.c abort.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/ref_build.sh).
 */
#ifndef TSU_REF_STUB_WAVEFRONT_ALIGN_H
#define TSU_REF_STUB_WAVEFRONT_ALIGN_H

typedef enum { indel = 0, edit = 1, gap_linear = 2, gap_affine = 3, gap_affine_2p = 4 } distance_metric_t;

typedef struct {
  int mismatch;
  int gap_opening;
  int gap_extension;
} affine_penalties_t;

typedef struct {
  distance_metric_t distance_metric;
  affine_penalties_t affine_penalties;
} wavefront_aligner_attr_t;

typedef struct {
  int score;
} cigar_t;

typedef struct {
  cigar_t* cigar;
} wavefront_aligner_t;

extern wavefront_aligner_attr_t wavefront_aligner_attr_default;
wavefront_aligner_t* wavefront_aligner_new(wavefront_aligner_attr_t* attributes);
int wavefront_align(wavefront_aligner_t* wf_aligner, const char* pattern, int pattern_length, const char* text,
                    int text_length);

#endif
