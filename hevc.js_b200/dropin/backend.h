// backend.h — the GPU back end a hevc::Decoder reconstructs through (internal to
// libhevcdec_gpu.so).
//
// A Backend belongs to one decoder, found from the DecodingContext the reference's hooks
// receive by the address of the decoder's DPB (ctx.dpb).  hooks.cpp records each picture's
// syntax into it and, at the end of the picture, hands the records to the GPU; the
// reconstructed samples are written back into the reference's Picture planes.
#pragma once

#include <cstdint>

namespace hevc {
class DPB;
struct Picture;
}  // namespace hevc

namespace dropin {

class Backend;

// The backend of the decoder that owns `dpb`, made on first use.  With `deferred`, the
// pictures go to the GPU on a worker thread while the next picture is parsed, and their
// samples are only guaranteed in host memory after finish(); without it (the default for
// a hevc::Decoder used directly, as the reference's CLI does) each picture's samples are
// in its planes when apply_sao returns.
Backend* attach(const hevc::DPB* dpb, bool deferred);
// Waits for the backend's work and frees it and its GPU context.
void detach(Backend* b);
// Waits until every picture handed to the GPU is written back.  0, or -1 after a failure
// (the message stays in last_error).
int finish(Backend* b);
const char* last_error(Backend* b);
int set_device(Backend* b, int device);
// Whether the GPU reconstructed this picture (its planes hold the GPU's samples).
bool reconstructed(Backend* b, const hevc::Picture* pic);
void stats(Backend* b, uint64_t* pictures, uint64_t* launches);
// Nanoseconds the decoder's calling threads have spent waiting for the back end: for room
// in the worker's queue, or for pictures to be written back.
uint64_t wait_ns(Backend* b);

}  // namespace dropin
