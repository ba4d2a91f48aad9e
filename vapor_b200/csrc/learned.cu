// Host side of the learned warm start (see unet.hpp for the architecture).
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "unet.hpp"

namespace vb {
namespace unet {

long weight_offset(int layer) {
    long off = 0;
    for (int l = 0; l < layer; ++l) off += 27L * kLayers[l].cout * kLayers[l].cin + kLayers[l].cout;
    return off;
}
long bias_offset(int layer) { return weight_offset(layer) + 27L * kLayers[layer].cout * kLayers[layer].cin; }
long head_offset() { return weight_offset(kConvLayers); }
long parameter_count() { return head_offset() + kHeadIn + 1; }

namespace {
__nv_bfloat16* bf(DevArray<uint16_t>& a) { return reinterpret_cast<__nv_bfloat16*>(a.p); }
}  // namespace

UNet::UNet(cudaStream_t stream) : s_(stream), own_(stream) {
    configure_conv_kernels();
    const long P = parameter_count();
    params_.allocate(P);
    grad_.allocate(P);
    m_.allocate(P);
    v_.allocate(P);
    wbf_.allocate(P);
    wpack_.allocate(P);
    long maxw = 0;
    for (const auto& l : kLayers) maxw = std::max(maxw, 27L * l.cout * l.cin);
    wflip_.allocate(maxw);
    partial_.allocate(1184);
    scalars_.allocate(8);
    scale_.allocate(1);
    error_.allocate(1);
    VB_CUDA(cudaMemsetAsync(error_.p, 0, sizeof(uint32_t), s_));
    init_parameters(1234u);
}

UNet::~UNet() { cudaStreamSynchronize(s_); }

void UNet::init_parameters(unsigned seed) {
    const long P = parameter_count();
    std::vector<float> h(P, 0.f);
    std::mt19937 rng(seed);
    for (int l = 0; l < kConvLayers; ++l) {
        const int cin_real = l == 0 ? 2 : kLayers[l].cin;
        const float bound = std::sqrt(6.f / float(27 * cin_real));
        std::uniform_real_distribution<float> U(-bound, bound);
        const long off = weight_offset(l);
        for (int tap = 0; tap < 27; ++tap)
            for (int co = 0; co < kLayers[l].cout; ++co)
                for (int ci = 0; ci < kLayers[l].cin; ++ci)
                    h[off + (long(tap) * kLayers[l].cout + co) * kLayers[l].cin + ci] =
                        (l == 0 && ci >= 2) ? 0.f : U(rng);
    }
    std::uniform_real_distribution<float> Uh(-0.25f, 0.25f);
    for (int c = 0; c < kHeadIn; ++c) h[head_offset() + c] = Uh(rng);
    set_parameters(h.data());
    step_ = 0;
}

void UNet::set_parameters(const float* host) {
    const long P = parameter_count();
    VB_CUDA(cudaMemcpyAsync(params_.p, host, P * sizeof(float), cudaMemcpyHostToDevice, s_));
    launch_to_bf16(P, params_.p, bf(wbf_), s_);
    pack_weights();
    m_.zero(s_);
    v_.zero(s_);
    VB_CUDA(cudaStreamSynchronize(s_));
    step_ = 0;
}

void UNet::get_parameters(float* host) {
    VB_CUDA(cudaMemcpyAsync(host, params_.p, parameter_count() * sizeof(float), cudaMemcpyDeviceToHost, s_));
    VB_CUDA(cudaStreamSynchronize(s_));
}

unsigned int UNet::error_flag() {
    uint32_t e = 0;
    VB_CUDA(cudaMemcpyAsync(&e, error_.p, sizeof(e), cudaMemcpyDeviceToHost, s_));
    VB_CUDA(cudaStreamSynchronize(s_));
    return e;
}

void UNet::check_error() {
    const unsigned int e = error_flag();
    if (!e) return;
    VB_CUDA(cudaMemsetAsync(error_.p, 0, sizeof(uint32_t), s_));
    VB_CUDA(cudaStreamSynchronize(s_));
    if (e & 2u)
        fail(VAPOR_RUNTIME_ERROR, "tensor-core convolution timed out and its in-flight MMAs could not be drained; "
                                  "tear down the CUDA context");
    fail(VAPOR_RUNTIME_ERROR, "tensor-core convolution timed out");
}

void UNet::ensure(int n) {
    if (n == n_) return;
    if (n % 4 != 0 || n < 8) fail(VAPOR_INVALID_ARGUMENT, "the warm-start network needs n divisible by 4 (n >= 8)");
    VB_CUDA(cudaStreamSynchronize(s_));
    const size_t V1 = size_t(n) * n * n, V2 = V1 / 8, V3 = V1 / 64;
    in0_.allocate(V1 * 16);
    e1a_.allocate(V1 * 16);
    dec1_.allocate(V1 * 48);
    e2in_.allocate(V2 * 16);
    e2a_.allocate(V2 * 32);
    dec2_.allocate(V2 * 96);
    e3in_.allocate(V3 * 32);
    e3a_.allocate(V3 * 64);
    e3b_.allocate(V3 * 64);
    d2a_.allocate(V2 * 32);
    d2b_.allocate(V2 * 32);
    d1a_.allocate(V1 * 16);
    d1b_.allocate(V1 * 16);
    out_.allocate(V1);
    n_ = n;
    ++generation_;
    // training buffers are allocated on first use (train_step)
    g1_.release();
    g2_.release();
    g3_.release();
    g4_.release();
    target_.release();
    gout_.release();
}

// The plane-window kernels' image of every layer's BF16 weights, at the
// layers' offsets in wbf_ (refreshed whenever wbf_ changes).
void UNet::pack_weights() {
    for (int l = 0; l < kConvLayers; ++l)
        launch_pack_window(kLayers[l].cout, kLayers[l].cin, bf(wbf_) + weight_offset(l), bf(wpack_) + weight_offset(l),
                           s_);
}

void UNet::conv(int layer, int D, int H, int W, const __nv_bfloat16* in, int in_stride, void* out, int out_stride,
                int out_offset, bool relu, bool fp32_out) {
    ConvArgs a{};
    a.D = D;
    a.H = H;
    a.W = W;
    a.in = in;
    a.in_stride = in_stride;
    a.cin = kLayers[layer].cin;
    a.w = bf(wbf_) + weight_offset(layer);
    a.bias = params_.p + bias_offset(layer);
    a.out = out;
    a.out_stride = out_stride;
    a.out_offset = out_offset;
    a.out_fp32 = fp32_out ? 1 : 0;
    a.relu = relu ? 1 : 0;
    a.error = error_.p;
    a.wait_probe = wait_probe_;
    a.w_window = bf(wpack_) + weight_offset(layer);
    launch_conv3(a, kLayers[layer].cout, s_);
}

void UNet::forward(int n) {
    const int h = n / 2, q = n / 4;
    const long V1 = long(n) * n * n;
    conv(0, n, n, n, bf(in0_), 16, e1a_.p, 16, 0, true);
    conv(1, n, n, n, bf(e1a_), 16, dec1_.p, 48, 32, true);  // skip 1 -> dec1[:, 32:48]
    launch_avgpool2(n, n, n, 16, bf(dec1_) + 32, 48, bf(e2in_), s_);
    conv(2, h, h, h, bf(e2in_), 16, e2a_.p, 32, 0, true);
    conv(3, h, h, h, bf(e2a_), 32, dec2_.p, 96, 64, true);  // skip 2 -> dec2[:, 64:96]
    launch_avgpool2(h, h, h, 32, bf(dec2_) + 64, 96, bf(e3in_), s_);
    conv(4, q, q, q, bf(e3in_), 32, e3a_.p, 64, 0, true);
    conv(5, q, q, q, bf(e3a_), 64, e3b_.p, 64, 0, true);
    launch_upsample2(q, q, q, 64, bf(e3b_), bf(dec2_), 96, s_);
    conv(6, h, h, h, bf(dec2_), 96, d2a_.p, 32, 0, true);
    conv(7, h, h, h, bf(d2a_), 32, d2b_.p, 32, 0, true);
    launch_upsample2(h, h, h, 32, bf(d2b_), bf(dec1_), 48, s_);
    conv(8, n, n, n, bf(dec1_), 48, d1a_.p, 16, 0, true);
    conv(9, n, n, n, bf(d1a_), 16, d1b_.p, 16, 0, true);
    launch_head(V1, kHeadIn, bf(d1b_), params_.p + head_offset(), params_.p + head_offset() + kHeadIn, out_.p, s_);
    VB_CUDA(cudaGetLastError());
}

void UNet::infer_into(int n, const float* b_split, const ProjControl* ctrl, float* x_split, double* x64_split) {
    ensure(n);
    launch_prep_input(n, b_split, ctrl, partial_.p, scale_.p, bf(in0_), s_);
    forward(n);
    launch_store_warm_start(n, out_.p, b_split, ctrl, partial_.p, scalars_.p, x_split, x64_split, s_);
    VB_CUDA(cudaGetLastError());
}

const float* UNet::precondition(int n, const float* rhs) {
    ensure(n);
    launch_prep_natural(long(n) * n * n, rhs, partial_.p, scalars_.p, scale_.p, bf(in0_), s_);
    forward(n);
    return out_.p;
}

void UNet::forward_features(int n, const __nv_bfloat16* input16, float* out) {
    ensure(n);
    const long V1 = long(n) * n * n;
    VB_CUDA(cudaMemcpyAsync(in0_.p, input16, V1 * 16 * sizeof(uint16_t), cudaMemcpyDeviceToDevice, s_));
    forward(n);
    VB_CUDA(cudaMemcpyAsync(out, out_.p, V1 * sizeof(float), cudaMemcpyDeviceToDevice, s_));
}

// Backward of one 3x3x3 layer: weight and bias gradients from (g, x); when
// dx is given, the input gradient dx = conv(g, flipped weights).
static void layer_backward(UNet& net, int layer, int D, int H, int W, const __nv_bfloat16* g, int g_stride,
                           int g_offset, const __nv_bfloat16* x, int x_stride, __nv_bfloat16* dx, int dx_stride,
                           int dx_offset, float* grad, __nv_bfloat16* wbf, __nv_bfloat16* wflip,
                           unsigned int* error, cudaStream_t s) {
    const int cin = kLayers[layer].cin, cout = kLayers[layer].cout;
    const long V = long(D) * H * W;
    WGradArgs wa{};
    wa.D = D;
    wa.H = H;
    wa.W = W;
    wa.g = g;
    wa.g_stride = g_stride;
    wa.g_offset = g_offset;
    wa.x = x;
    wa.x_stride = x_stride;
    wa.cout = cout;
    wa.cin = cin;
    wa.dw = grad + weight_offset(layer);
    wa.error = error;
    launch_conv3_wgrad(wa, s);
    launch_bias_grad(V, cout, g, g_stride, g_offset, grad + bias_offset(layer), s);
    if (!dx) return;
    launch_flip_weights(cout, cin, wbf + weight_offset(layer), wflip, s);
    ConvArgs a{};
    a.D = D;
    a.H = H;
    a.W = W;
    a.in = g + g_offset;
    a.in_stride = g_stride;
    a.cin = cout;
    a.w = wflip;
    a.bias = nullptr;
    a.out = dx;
    a.out_stride = dx_stride;
    a.out_offset = dx_offset;
    a.out_fp32 = 0;
    a.relu = 0;
    a.error = error;
    launch_conv3(a, cin, s);
    (void)net;
}

void UNet::backward(int n) {
    const int h = n / 2, q = n / 4;
    const long V1 = long(n) * n * n, V2 = V1 / 8, V3 = V1 / 64;
    if (g1_.n != size_t(V1) * 48) {
        g1_.allocate(size_t(V1) * 48);  // dec1 gradient [V1][48]
        g2_.allocate(size_t(V1) * 32);  // two level-1 gradients [V1][16]
        g3_.allocate(size_t(V2) * 96);  // dec2 gradient [V2][96]
        g4_.allocate(size_t(V2) * 64 + size_t(V3) * 128);
    }
    __nv_bfloat16* gdec1 = bf(g1_);
    __nv_bfloat16* gA = bf(g2_);                   // [V1][16]
    __nv_bfloat16* gB = gA + size_t(V1) * 16;      // [V1][16]
    __nv_bfloat16* gdec2 = bf(g3_);
    __nv_bfloat16* gl2 = bf(g4_);                  // [V2][32]
    __nv_bfloat16* gl2b = gl2 + size_t(V2) * 32;   // [V2][32]
    __nv_bfloat16* gl3a = gl2b + size_t(V2) * 32;  // [V3][64]
    __nv_bfloat16* gl3b = gl3a + size_t(V3) * 64;  // [V3][64]
    float* grad = grad_.p;
    __nv_bfloat16* wb = bf(wbf_);
    __nv_bfloat16* wf = bf(wflip_);
    unsigned int* err = error_.p;

    // head: d(d1b) = g * w_head, masked by the ReLU of layer 9
    launch_head_backward(V1, kHeadIn, bf(d1b_), params_.p + head_offset(), gout_.p, gA, grad + head_offset(),
                         grad + head_offset() + kHeadIn, s_);
    // layer 9 (input d1a)
    layer_backward(*this, 9, n, n, n, gA, 16, 0, bf(d1a_), 16, gB, 16, 0, grad, wb, wf, err, s_);
    launch_relu_mask(V1, 16, bf(d1a_), 16, 0, gB, 16, 0, s_);
    // layer 8 (input dec1 = [upsample(d2b) : 32 | skip1 : 16])
    layer_backward(*this, 8, n, n, n, gB, 16, 0, bf(dec1_), 48, gdec1, 48, 0, grad, wb, wf, err, s_);
    launch_upsample2_backward(h, h, h, 32, gdec1, 48, gl2b, s_);
    launch_relu_mask(V2, 32, bf(d2b_), 32, 0, gl2b, 32, 0, s_);
    // layer 7 (input d2a)
    layer_backward(*this, 7, h, h, h, gl2b, 32, 0, bf(d2a_), 32, gl2, 32, 0, grad, wb, wf, err, s_);
    launch_relu_mask(V2, 32, bf(d2a_), 32, 0, gl2, 32, 0, s_);
    // layer 6 (input dec2 = [upsample(e3b) : 64 | skip2 : 32])
    layer_backward(*this, 6, h, h, h, gl2, 32, 0, bf(dec2_), 96, gdec2, 96, 0, grad, wb, wf, err, s_);
    launch_upsample2_backward(q, q, q, 64, gdec2, 96, gl3b, s_);
    launch_relu_mask(V3, 64, bf(e3b_), 64, 0, gl3b, 64, 0, s_);
    // layer 5 (input e3a)
    layer_backward(*this, 5, q, q, q, gl3b, 64, 0, bf(e3a_), 64, gl3a, 64, 0, grad, wb, wf, err, s_);
    launch_relu_mask(V3, 64, bf(e3a_), 64, 0, gl3a, 64, 0, s_);
    // layer 4 (input e3in = pool(skip2)); its input gradient reuses gl3b as [V3][32]
    layer_backward(*this, 4, q, q, q, gl3a, 64, 0, bf(e3in_), 32, gl3b, 32, 0, grad, wb, wf, err, s_);
    launch_avgpool2_backward(h, h, h, 32, gl3b, gdec2, 96, 64, true, s_);
    launch_relu_mask(V2, 32, bf(dec2_), 96, 64, gdec2, 96, 64, s_);
    // layer 3 (input e2a), output gradient gdec2[:, 64:96]
    layer_backward(*this, 3, h, h, h, gdec2, 96, 64, bf(e2a_), 32, gl2, 32, 0, grad, wb, wf, err, s_);
    launch_relu_mask(V2, 32, bf(e2a_), 32, 0, gl2, 32, 0, s_);
    // layer 2 (input e2in = pool(skip1)); its input gradient reuses gl2b as [V2][16]
    layer_backward(*this, 2, h, h, h, gl2, 32, 0, bf(e2in_), 16, gl2b, 16, 0, grad, wb, wf, err, s_);
    launch_avgpool2_backward(n, n, n, 16, gl2b, gdec1, 48, 32, true, s_);
    launch_relu_mask(V1, 16, bf(dec1_), 48, 32, gdec1, 48, 32, s_);
    // layer 1 (input e1a), output gradient gdec1[:, 32:48]
    layer_backward(*this, 1, n, n, n, gdec1, 48, 32, bf(e1a_), 16, gA, 16, 0, grad, wb, wf, err, s_);
    launch_relu_mask(V1, 16, bf(e1a_), 16, 0, gA, 16, 0, s_);
    // layer 0 (input features): no input gradient needed
    layer_backward(*this, 0, n, n, n, gA, 16, 0, bf(in0_), 16, nullptr, 0, 0, grad, wb, wf, err, s_);
    VB_CUDA(cudaGetLastError());
}

void UNet::backward_from_output(int n, const float* grad_out) {
    ensure(n);
    const long V1 = long(n) * n * n;
    if (gout_.n != size_t(V1)) gout_.allocate(V1);
    VB_CUDA(cudaMemcpyAsync(gout_.p, grad_out, V1 * sizeof(float), cudaMemcpyDeviceToDevice, s_));
    grad_.zero(s_);
    backward(n);
}

double UNet::train_step(int n, const float* b_split, const float* p_split, const ProjControl* ctrl, float lr) {
    ensure(n);
    const long V1 = long(n) * n * n;
    if (target_.n != size_t(V1)) {
        target_.allocate(V1);
        gout_.allocate(V1);
    }
    launch_prep_input(n, b_split, ctrl, partial_.p, scale_.p, bf(in0_), s_);
    launch_target(n, p_split, ctrl, scale_.p, target_.p, s_);
    forward(n);
    launch_loss_grad(V1, out_.p, target_.p, partial_.p, scalars_.p, gout_.p, s_);
    double loss = 0.0;
    VB_CUDA(cudaMemcpyAsync(&loss_host_, scalars_.p + 2, sizeof(double), cudaMemcpyDeviceToHost, s_));
    grad_.zero(s_);
    backward(n);
    ++step_;
    launch_adam(parameter_count(), params_.p, m_.p, v_.p, grad_.p, bf(wbf_), lr, step_, s_);
    pack_weights();
    VB_CUDA(cudaStreamSynchronize(s_));
    check_error();
    loss = loss_host_;
    return loss;
}

double UNet::evaluate(int n, const float* b_split, const float* p_split, const ProjControl* ctrl) {
    ensure(n);
    const long V1 = long(n) * n * n;
    if (target_.n != size_t(V1)) {
        target_.allocate(V1);
        gout_.allocate(V1);
    }
    launch_prep_input(n, b_split, ctrl, partial_.p, scale_.p, bf(in0_), s_);
    launch_target(n, p_split, ctrl, scale_.p, target_.p, s_);
    forward(n);
    launch_loss_grad(V1, out_.p, target_.p, partial_.p, scalars_.p, nullptr, s_);
    VB_CUDA(cudaMemcpyAsync(&loss_host_, scalars_.p + 2, sizeof(double), cudaMemcpyDeviceToHost, s_));
    VB_CUDA(cudaStreamSynchronize(s_));
    check_error();
    return loss_host_;
}

}  // namespace unet
}  // namespace vb
