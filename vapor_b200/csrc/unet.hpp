// Learned warm start for the pressure solve: a 3-level 3D U-Net mapping the
// normalized divergence (and a solid mask) to the normalized pressure.
//
//   level 1 (n^3):      conv 16->16, conv 16->16          (input: 2 real channels padded to 16)
//   level 2 ((n/2)^3):  avgpool, conv 16->32, conv 32->32
//   level 3 ((n/4)^3):  avgpool, conv 32->64, conv 64->64
//   decoder 2:          upsample 64 ++ skip 32 = 96 -> conv 96->32, conv 32->32
//   decoder 1:          upsample 32 ++ skip 16 = 48 -> conv 48->16, conv 16->16
//   head:               1x1 conv 16->1 (FP32 output)
// ReLU after every 3x3x3 convolution; about 0.35 M parameters; BF16 weights
// and activations, FP32 accumulation, FP32 master weights and Adam state.
// The problem is linear in the divergence, so inputs and targets are divided
// by the RMS of the mean-free right-hand side and outputs multiplied back.
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "engine.hpp"

namespace vb {
namespace unet {

struct ConvArgs {
    int D, H, W;                  // grid (z, y, x)
    const __nv_bfloat16* in;      // channels-last, in_stride channels per voxel
    int in_stride;
    int cin;                      // multiple of 16
    const __nv_bfloat16* w;       // [27][cout][cin], tap = (dz+1)*9 + (dy+1)*3 + (dx+1)
    const float* bias;            // [cout] or null
    void* out;                    // BF16 or FP32, out_stride channels per voxel
    int out_stride;
    int out_offset;
    int out_fp32;
    int relu;
    unsigned int* error;          // bit 1: a bounded wait timed out; bit 2: in-flight MMAs could not be drained
    int wait_probe;               // test hook: > 0 makes each CTA's first completion wait poll a barrier
                                  // that nothing completes, wait_probe times, so that it runs out
    const __nv_bfloat16* w_window;  // w packed for the plane-window kernels (launch_pack_window), or null
};

struct WGradArgs {
    int D, H, W;
    const __nv_bfloat16* g;  // output gradient, channels-last
    int g_stride, g_offset;
    const __nv_bfloat16* x;  // layer input, channels-last
    int x_stride;
    int cout, cin;           // multiples of 16
    float* dw;               // [27][cout][cin], accumulated
    unsigned int* error;     // tensor-core form: bit 1 a bounded wait timed out (may be null for the other form)
};

// Sets the kernels' shared-memory limits (once per device, before use).
void configure_conv_kernels();
// Selects the kernel of every later convolution whose weights fit in shared
// memory: 0 the block-synchronous z-march, 1 its warp-specialised form (same
// results), 2 the plane-window form (same results with one input chunk,
// FP32-rounding differences with several), 3 the plane-window form fed by TMA
// (the same MMAs as 2, so the same results; needs ConvArgs::w_window, else 2
// runs).
void set_conv_kernel(int kind);
// Packs one layer's weights [27][cout][cin] into the shared-memory image of
// the plane-window kernels (27 cout cin values).
void launch_pack_window(int cout, int cin, const __nv_bfloat16* w, __nv_bfloat16* packed, cudaStream_t s);
void launch_conv3(const ConvArgs& a, int cout, cudaStream_t s);
void launch_conv3_wgrad(const WGradArgs& a, cudaStream_t s);
// Weight-gradient kernel: 1 (default) tcgen05 implicit GEMM, 0 the CUDA-core
// form. Both accumulate FP32 products of the same BF16 values with atomics,
// so they agree to FP32 rounding.
void set_wgrad_kernel(int kind);
void launch_prep_input(int n, const float* b_split, const ProjControl* ctrl, double* partial, float* scale,
                       __nv_bfloat16* out, cudaStream_t s);
// Features from a natural-layout FP32 field: channel 0 = (a - mean) / rms.
// Uses partial[0..1183], scalars[0].
void launch_prep_natural(long V, const float* a, double* partial, double* scalars, float* scale,
                         __nv_bfloat16* out, cudaStream_t s);
void launch_avgpool2(int D, int H, int W, int C, const __nv_bfloat16* in, int in_stride, __nv_bfloat16* out,
                     cudaStream_t s);
void launch_upsample2(int d, int h, int w, int C, const __nv_bfloat16* in, __nv_bfloat16* out, int out_stride,
                      cudaStream_t s);
void launch_head(long V, int C, const __nv_bfloat16* act, const float* w, const float* bias, float* out,
                 cudaStream_t s);
void launch_mean(long V, const float* a, double* partial, double* mean, cudaStream_t s);
// x = alpha (p - mean p) into the solver's split iterate (FP32 or FP64), alpha
// by the Galerkin condition against the mean-free right-hand side. Uses
// partial[0..1183] and scalars[0..1].
void launch_store_warm_start(int n, const float* p, const float* b_split, const ProjControl* ctrl,
                             double* partial, double* scalars, float* x_split, double* x64_split, cudaStream_t s);
void launch_target(int n, const float* p_split, const ProjControl* ctrl, const float* scale, float* target,
                   cudaStream_t s);
// Scale-invariant loss 1 - cos^2(p - mean p, t - mean t) into scalars[2] and,
// when grad is given, its gradient with respect to p. Uses scalars[0..4].
void launch_loss_grad(long V, const float* p, const float* t, double* partial, double* scalars, float* grad,
                      cudaStream_t s);
void launch_head_backward(long V, int C, const __nv_bfloat16* act, const float* w, const float* g,
                          __nv_bfloat16* dact, float* dw, float* db, cudaStream_t s);
void launch_relu_mask(long V, int C, const __nv_bfloat16* act, int act_stride, int act_offset, __nv_bfloat16* g,
                      int g_stride, int g_offset, cudaStream_t s);
void launch_bias_grad(long V, int C, const __nv_bfloat16* g, int g_stride, int g_offset, float* db, cudaStream_t s);
void launch_flip_weights(int cout, int cin, const __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t s);
void launch_avgpool2_backward(int D, int H, int W, int C, const __nv_bfloat16* dout, __nv_bfloat16* din,
                              int din_stride, int din_offset, bool add, cudaStream_t s);
void launch_upsample2_backward(int d, int h, int w, int C, const __nv_bfloat16* dfine, int fine_stride,
                               __nv_bfloat16* dcoarse, cudaStream_t s);
void launch_adam(long count, float* w, float* m, float* v, const float* g, __nv_bfloat16* wb, float lr, int step,
                 cudaStream_t s);
void launch_to_bf16(long count, const float* a, __nv_bfloat16* b, cudaStream_t s);

// Parameter block layout: 10 convolutions (3x3x3) then the head.
struct LayerShape {
    int cin, cout;
};
constexpr int kConvLayers = 10;
constexpr LayerShape kLayers[kConvLayers] = {{16, 16}, {16, 16}, {16, 32}, {32, 32}, {32, 64},
                                             {64, 64}, {96, 32}, {32, 32}, {48, 16}, {16, 16}};
constexpr int kHeadIn = 16;

// All trainable parameters in one FP32 vector: for each conv layer its
// weights [27][cout][cin] then its bias [cout]; then head weights [16] and
// head bias [1].
long parameter_count();
long weight_offset(int layer);
long bias_offset(int layer);
long head_offset();

class UNet {
public:
    explicit UNet(cudaStream_t stream);
    ~UNet();
    // The stream all later work is ordered on (the owning simulation's while
    // a simulation uses the network, else the one given at construction).
    void set_stream(cudaStream_t s) { s_ = s; }
    void use_own_stream() { s_ = own_; }
    cudaStream_t stream() const { return s_; }
    // Allocates the activation buffers for n (outside any stream capture).
    void prepare(int n) { ensure(n); }
    // Incremented whenever the activation buffers are reallocated; a recorded
    // CUDA graph that uses the network is valid only for one generation.
    unsigned long long generation() const { return generation_; }
    UNet(const UNet&) = delete;
    UNet& operator=(const UNet&) = delete;

    void set_parameters(const float* host);  // parameter_count() floats
    void get_parameters(float* host);
    void init_parameters(unsigned seed);      // He-uniform weights, zero biases

    // Forward on an n^3 grid (n divisible by 4) from the solver's split RHS;
    // writes the warm start x = alpha * (p - mean p) into x_split (FP32) or
    // x64_split (FP64), alpha = (q.b)/(q.Aq) for q = p - mean p. Errors raise.
    void infer_into(int n, const float* b_split, const ProjControl* ctrl, float* x_split, double* x64_split);
    // One training step on (b, p*) from a finished projection: forward,
    // loss, backward, Adam. Returns the loss (waits for the device).
    double train_step(int n, const float* b_split, const float* p_split, const ProjControl* ctrl, float lr);
    // Forward only and the loss against p* (no update); waits. The loss is
    // the relative squared error left after the best scaling of the
    // prediction, 1 - cos^2 between the mean-free prediction and p*.
    double evaluate(int n, const float* b_split, const float* p_split, const ProjControl* ctrl);
    unsigned int error_flag();
    // Waits for the network's stream, then raises VAPOR_RUNTIME_ERROR if a
    // tensor-core wait ran out since the last check (clearing the flag, so
    // later calls start clean). When in-flight MMAs could not be drained as
    // well, the message says the CUDA context must be torn down.
    void check_error();
    // Test hook for the timeout path: > 0 makes the next convolutions' first
    // completion wait poll a barrier that nothing completes, `iterations`
    // times; 0 restores normal waits.
    void set_wait_probe(int iterations) { wait_probe_ = iterations; }
    int adam_steps() const { return step_; }
    // Raw forward on device channels-last input [n^3][16] -> FP32 output.
    void forward_features(int n, const __nv_bfloat16* input16, float* out);
    void backward_from_output(int n, const float* grad_out);  // after forward_features
    // Coarse-grid correction of the flexible PCG solve: the network applied
    // to a natural-layout FP32 right-hand side on an n^3 grid; returns the
    // FP32 output (natural layout, valid until the next call). Its scale is
    // arbitrary: the caller scales it by the Galerkin condition.
    const float* precondition(int n, const float* rhs);
    float* gradient() { return grad_.p; }

private:
    void ensure(int n);
    void forward(int n);
    void backward(int n);
    void pack_weights();
    void conv(int layer, int D, int H, int W, const __nv_bfloat16* in, int in_stride, void* out, int out_stride,
              int out_offset, bool relu, bool fp32_out = false);

    cudaStream_t s_;
    cudaStream_t own_;
    int n_ = 0;
    int step_ = 0;
    unsigned long long generation_ = 0;
    DevArray<float> params_, grad_, m_, v_;
    DevArray<uint16_t> wbf_;   // BF16 copy of the parameters
    DevArray<uint16_t> wpack_;  // wbf_'s weights packed for the plane-window kernels (same offsets)
    DevArray<uint16_t> wflip_;  // flipped/transposed weights of one layer
    // activations (BF16, channels-last)
    DevArray<uint16_t> in0_, e1a_, dec1_, e2in_, e2a_, dec2_, e3in_, e3a_, e3b_, d2a_, d2b_, d1a_, d1b_;
    // gradients (BF16)
    DevArray<uint16_t> g1_, g2_, g3_, g4_;
    DevArray<float> out_, target_, gout_;
    double loss_host_ = 0.0;
    DevArray<double> partial_, scalars_;
    DevArray<float> scale_;
    DevArray<uint32_t> error_;
    int wait_probe_ = 0;
};

}  // namespace unet
}  // namespace vb
