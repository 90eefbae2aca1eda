// A finished batch recording handed from the batch (avbd_batch.cu) to the adjoint (avbd_adjoint.cu):
// the device arrays as avbd_record.cu wrote them, which the adjoint adopts, and the host copy of
// the bodies when recording started.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "avbd.h"

namespace avbd {

struct RecordingHandoff {
  int device = 0;
  uint32_t K = 0, W = 0, nb = 0, maxPts = 0;
  uint64_t manifolds = 0, points = 0;
  // device arrays (layout of RecordDev): K x (W + 1) first indices, per manifold bodies (int2) and
  // basis (9 doubles), per point anchors (6 doubles), manifold and source, K x nb colours, K x W counts
  const int *manFirst = nullptr, *ptFirst = nullptr, *ptMan = nullptr, *ptPrev = nullptr, *color = nullptr, *ncol = nullptr;
  const void* manAB = nullptr;
  const double *basis = nullptr, *anchors = nullptr;
  std::vector<void*> mem;             // every device allocation of the recording: the receiver frees them
  std::vector<uint32_t> worldFirst;   // W + 1
  std::vector<avbd_body> initial;     // the bodies when recording started
  avbd_params params{};
};

// Moves a complete recording out of the batch (the batch no longer holds it); on failure `why`
// says what is missing and the recording stays with the batch.
int batch_take_recording(avbd_batch* b, RecordingHandoff& out, std::string& why);

}  // namespace avbd
