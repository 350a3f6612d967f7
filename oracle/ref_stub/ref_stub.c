/* Definitions behind oracle/ref_stub/wavefront/wavefront_align.h: they exist
 * so the reference's wfa_gpu.cu links; its check=1 branch never runs under
 * the harness.  TEST INFRASTRUCTURE ONLY. */
#include <stdio.h>
#include <stdlib.h>

#include "wavefront/wavefront_align.h"

wavefront_aligner_attr_t wavefront_aligner_attr_default = {gap_affine, {4, 6, 2}};

wavefront_aligner_t* wavefront_aligner_new(wavefront_aligner_attr_t* attributes) {
  (void)attributes;
  fprintf(stderr, "ref_stub: WFA2-lib is not available\n");
  abort();
}

int wavefront_align(wavefront_aligner_t* wf_aligner, const char* pattern, int pattern_length, const char* text,
                    int text_length) {
  (void)wf_aligner, (void)pattern, (void)pattern_length, (void)text, (void)text_length;
  fprintf(stderr, "ref_stub: WFA2-lib is not available\n");
  abort();
}
