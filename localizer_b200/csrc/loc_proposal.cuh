// Host-side interface of the learned start proposal (used by the fit
// pipeline to warm-start the solver).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

struct loc_proposal;

namespace locb {

// Device view of a proposal network: FP32 master weights and the packed
// BF16 tensor-core operands of its two 3x3 convolutions.
struct ProposalView {
    int nout;          // parameters it proposes: 5 (symmetric), 4 (fixed width), 7 (ellipsoidal)
    int device;
    const float *w;    // master weights
    const void *wp;    // packed BF16 operands (conv2 then conv3)
    int *err;          // set to 1 if a tensor-core wait ran out
};

int proposal_nout(int method);  // 5 / 4 / 7, or 0 for an unsupported method
bool proposal_view(const loc_proposal *p, ProposalView *v);

// Enqueue the network over every candidate and the start check. For each
// candidate i, init[i*P .. i*P+P) receives the proposed parameter vector in
// absolute frame coordinates when the proposal's residual over the
// candidate's ROI is not worse than the solver's own cold start, else NaN in
// slot 0 (the solver then starts cold). Candidates with cls[i] < 0 (not
// fitted) get NaN. n_warm counts proposals taken.
cudaError_t enqueue_proposal(const ProposalView &net, const uint16_t *frames, long long frame_px, int n_rows,
                             int n_cols, const void *cands, const int *cls, int n, int method, float w0, float *init,
                             unsigned long long *n_warm, int *err, cudaStream_t stream, int *launches);

}  // namespace locb
