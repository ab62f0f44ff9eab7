// Learned short-range network: three valid 3x3x3 convolutions (16 channels,
// GELU) and a linear head 16 -> 3 read at the particles by trilinear (CIC)
// interpolation.  The convolutions run on the tcgen05 tensor cores in BF16
// with FP32 accumulation in tensor memory; the weight gradients, the head,
// the loss and Adam run on the CUDA cores in FP32.
//
// Tensors are channel-last BF16 volumes [B][Z][Y][X][16] (32 bytes a node);
// input channels beyond the network's c_in are zero.  No counterpart exists in
// the reference: the network's definition is the CPU restatement that the
// tests compare against (forward, gradients, Adam).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpm {
namespace cnn {

constexpr int CH = 16;                // hidden channels and the padded input width
constexpr int NOUT = 3;               // head outputs (acceleration components)
constexpr int MAX_CIN = 16;           // network input channels supported
constexpr int WPACK_U4 = 27 * 32;     // one packed layer: 27 taps x 16 x 16 bf16 = 13,824 bytes

// Offsets of the parts of the flat float32 parameter vector:
// [W1 (27,16,c_in), b1, W2 (27,16,16), b2, W3 (27,16,16), b3, Wh (3,16), bh (3)].
struct Layout {
  int c_in;
  int64_t w[3], b[3], wh, bh, total;
};
Layout layout(int c_in);

// Node dims of a batch of volumes.
struct Vol {
  int b, z, y, x;
  int64_t nodes() const { return (int64_t)b * z * y * x; }
};

// Packed weights of the three layers (forward) and of layers 2 and 3 with the
// taps flipped and the channels transposed (input gradient).
struct Packed {
  uint4* fwd[3];
  uint4* bwd[3];  // bwd[0] unused
};

// Valid convolution out[o] = GELU(bias + sum_t W[t] in[o + t]) with optional
// store of the pre-activation; output dims are the input's minus 2.
void conv_forward(const __nv_bfloat16* in, Vol vin, __nv_bfloat16* out, __nv_bfloat16* zout, const uint4* wpack,
                  const float* bias, uint32_t* err, cudaStream_t s);
// Input gradient of a convolution times GELU'(zprev): dzprev[i] =
// GELU'(zprev[i]) * sum_t W[t]^T dz[i - t] (a full convolution, dims + 2).
void conv_backward_data(const __nv_bfloat16* dz, Vol vdz, __nv_bfloat16* dzprev, const __nv_bfloat16* zprev,
                        const uint4* wpack_bwd, uint32_t* err, cudaStream_t s);
// Self-test of the tensor-core wait's time limit (one tile with no MMA issued,
// then a normal tile); returns the seconds the timed-out launch took.
double conv_wait_selftest(cudaStream_t s);
// Weight and bias gradients of a valid convolution (accumulated, FP32).
void conv_backward_weights(const __nv_bfloat16* x, Vol vin, const __nv_bfloat16* dz, int cin, float* dw, float* db,
                           cudaStream_t s);
// Pack the float32 parameters into the tensor-core operand layouts.
void pack_weights(const float* params, const Layout& L, const Packed& P, cudaStream_t s);

// Per-particle head read for inference: the acceleration (network units)
// at node coordinates (sx, sy, sz) of volume b.
struct HeadParticles {
  int64_t n;
  const int32_t* pb;   // volume index (nullptr: 0)
  const float* ps;     // n x 3 node coordinates local to the output volume
  float* out;          // n x 3
};
void head_at_particles(const __nv_bfloat16* a3, Vol v3, const float* params, const Layout& L,
                       const HeadParticles& hp, cudaStream_t s);
// The same read on a periodic volume (corner i + 1 wraps to 0).
void head_periodic(const __nv_bfloat16* a3, Vol v3, const float* params, const Layout& L, const HeadParticles& hp,
                   cudaStream_t s);
// Head output at every node (nodes x 3, FP32).
void head_field(const __nv_bfloat16* a3, int64_t nodes, const float* params, const Layout& L, float* out,
                cudaStream_t s);
// Weighted squared error of the interpolated head against targets: adds the
// loss to *loss and d loss / d (head output) to dout (nodes x 3).
void head_loss(const __nv_bfloat16* a3, Vol v3, const float* params, const Layout& L, int64_t n, const int32_t* pb,
               const float* ps, const float* tgt, const float* w, const float* wsum, float* dout, float* loss,
               cudaStream_t s);
// Head backward: dz3 from dout and the layer-3 pre-activation; adds the head's
// weight gradients to grad.
void head_backward(const __nv_bfloat16* a3, const __nv_bfloat16* z3, const float* dout, int64_t nodes,
                   const float* params, const Layout& L, __nv_bfloat16* dz3, float* grad, cudaStream_t s);
// One Adam step (step counts from 1) over n parameters.
void adam(float* p, float* m, float* v, const float* g, int64_t n, float lr, float b1, float b2, float eps,
          int64_t step, cudaStream_t s);

}  // namespace cnn
}  // namespace tpm
