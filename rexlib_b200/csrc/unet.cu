// The learned prior: a 3D U-Net of four levels (16, 32, 64, 128 channels;
// two 3x3x3 convolutions with ReLU a level, 2x2x2 mean pooling down, 2x2x2
// stride-2 transposed convolutions up, skip tensors concatenated in the
// decoder, a 1x1x1 head added to the input), about 1.4 million parameters.
// Forward and backward run on this library's own kernels: the 3x3x3
// convolutions and their input gradients on the tcgen05 tensor cores (the
// backward as a convolution with the flipped, transposed weights, its ReLU
// mask in the epilogue), the rest on the CUDA cores. Activations are BF16,
// sums FP32, parameters FP32 with BF16 copies for the tensor cores, trained
// with Adam. No counterpart in the reference (rexlib has no learned part).
#include "unet_kernels.cuh"
#include "conv3d.cuh"

#include <algorithm>
#include <cmath>
#include <random>
#include <string>
#include <vector>

namespace rexlib_b200
{
namespace unet
{
namespace
{

enum class layer_kind
{
	first,
	conv,
	up,
	head
};

struct layer_def
{
	layer_kind kind;
	int cin_a, cin_b, cout;
};

// The network, encoder to decoder.
enum layer_id
{
	L_FIRST, L_E0, L_E1A, L_E1, L_E2A, L_E2, L_B1, L_B2, L_UP2, L_D2A, L_D2, L_UP1, L_D1A, L_D1, L_UP0, L_D0A, L_D0,
	L_HEAD, LAYERS
};

const layer_def defs[LAYERS] = {
	{layer_kind::first, 1, 0, 16},   {layer_kind::conv, 16, 0, 16},  {layer_kind::conv, 16, 0, 32},
	{layer_kind::conv, 32, 0, 32},   {layer_kind::conv, 32, 0, 64},  {layer_kind::conv, 64, 0, 64},
	{layer_kind::conv, 64, 0, 128},  {layer_kind::conv, 128, 0, 128}, {layer_kind::up, 128, 0, 64},
	{layer_kind::conv, 64, 64, 64},  {layer_kind::conv, 64, 0, 64},  {layer_kind::up, 64, 0, 32},
	{layer_kind::conv, 32, 32, 32},  {layer_kind::conv, 32, 0, 32},  {layer_kind::up, 32, 0, 16},
	{layer_kind::conv, 16, 16, 16},  {layer_kind::conv, 16, 0, 16},  {layer_kind::head, 16, 0, 1},
};

int64_t weight_count(const layer_def &l)
{
	const int cin = l.cin_a + l.cin_b;
	switch (l.kind)
	{
	case layer_kind::first:
		return 27LL * l.cout;
	case layer_kind::conv:
		return 27LL * l.cout * cin;
	case layer_kind::up:
		return 8LL * l.cout * cin;
	default:
		return cin;
	}
}

int64_t fan_in(const layer_def &l)
{
	const int cin = l.cin_a + l.cin_b;
	return l.kind == layer_kind::up ? cin : l.kind == layer_kind::head ? cin : 27LL * cin;
}

template <typename T>
T *device_alloc(size_t count)
{
	void *p = nullptr;
	check_cuda(cudaMalloc(&p, count * sizeof(T) + 16), "allocation of the prior's buffers");
	check_cuda(cudaMemset(p, 0, count * sizeof(T) + 16), "clearing the prior's buffers");
	return static_cast<T *>(p);
}

int grid_for(int64_t n, int threads = 256)
{
	const int64_t blocks = (n + threads - 1) / threads;
	return static_cast<int>(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

} // anonymous namespace

} // namespace unet
} // namespace rexlib_b200

struct rexlib_b200_unet
{
	int extent = 0;
	int64_t parameter_count = 0;
	int64_t weight_offset[rexlib_b200::unet::LAYERS] = {};
	int64_t bias_offset[rexlib_b200::unet::LAYERS] = {};
	float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
	__nv_bfloat16 *params16 = nullptr; // BF16 copies of every parameter (the convolutions read their weights)
	__nv_bfloat16 *flipped = nullptr;   // flipped, transposed weights of each 3x3x3 convolution
	int64_t flip_offset[rexlib_b200::unet::LAYERS] = {};
	int steps = 0;
	int *error = nullptr;
	// Activations: index = the layer producing it; pooled and upsampled ones besides.
	__nv_bfloat16 *act[rexlib_b200::unet::LAYERS] = {};
	__nv_bfloat16 *pooled[3] = {};
	__nv_bfloat16 *grad_a[rexlib_b200::unet::LAYERS] = {}; // gradient of each layer's output
	__nv_bfloat16 *grad_skip[3] = {};                      // gradient reaching a skip tensor from the decoder
	__nv_bfloat16 *grad_pooled[3] = {};
	const float *input = nullptr; // of the last forward
	float *output = nullptr;
	std::vector<void *> owned;
};

namespace rexlib_b200
{
namespace unet
{
namespace
{

using net_t = rexlib_b200_unet;

// The extent of the volume a layer produces: the encoder halves the input
// extent per level, the decoder doubles it back.
int level_of(int layer)
{
	switch (layer)
	{
	case L_FIRST:
	case L_E0:
	case L_UP0:
	case L_D0A:
	case L_D0:
	case L_HEAD:
		return 0;
	case L_E1A:
	case L_E1:
	case L_UP1:
	case L_D1A:
	case L_D1:
		return 1;
	case L_E2A:
	case L_E2:
	case L_UP2:
	case L_D2A:
	case L_D2:
		return 2;
	default:
		return 3;
	}
}

volume_shape shape_at(const net_t &n, int lvl)
{
	const int e = n.extent >> lvl;
	return volume_shape{e, e, e};
}

int64_t voxels_at(const net_t &n, int lvl)
{
	const int64_t e = n.extent >> lvl;
	return e * e * e;
}

void allocate(net_t &n)
{
	int64_t offset = 0;
	int64_t flip = 0;
	for (int l = 0; l < LAYERS; ++l)
	{
		n.weight_offset[l] = offset;
		offset += weight_count(defs[l]);
		n.bias_offset[l] = offset;
		offset += defs[l].cout;
		offset = (offset + 7) / 8 * 8; // 16-byte aligned BF16 copies
		if (defs[l].kind == layer_kind::conv)
		{
			n.flip_offset[l] = flip;
			flip += weight_count(defs[l]);
		}
	}
	n.parameter_count = offset;
	auto wgrad_smem = [](int cout) {
		return static_cast<int>(sizeof(float) * wgrad_chunk * (cout + 4 * wgrad_threads / (cout / 4)));
	};
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wgrad_smem(16)),
		"weight-gradient attributes");
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, wgrad_smem(32)),
		"weight-gradient attributes");
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, wgrad_smem(64)),
		"weight-gradient attributes");
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, wgrad_smem(128)),
		"weight-gradient attributes");
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				   wgrad_smem(128)),
		"weight-gradient attributes");
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				   wgrad_smem(256)),
		"weight-gradient attributes");
	check_cuda(cudaFuncSetAttribute(wgrad_kernel<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				   wgrad_smem(512)),
		"weight-gradient attributes");
	auto own = [&](auto *p) {
		n.owned.push_back(p);
		return p;
	};
	n.params = own(device_alloc<float>(offset));
	n.grads = own(device_alloc<float>(offset));
	n.adam_m = own(device_alloc<float>(offset));
	n.adam_v = own(device_alloc<float>(offset));
	n.params16 = own(device_alloc<bf16>(offset));
	n.flipped = own(device_alloc<bf16>(flip));
	n.error = own(device_alloc<int>(1));
	for (int l = 0; l < L_HEAD; ++l)
	{
		const int64_t v = voxels_at(n, level_of(l));
		n.act[l] = own(device_alloc<bf16>(v * defs[l].cout));
		n.grad_a[l] = own(device_alloc<bf16>(v * defs[l].cout));
	}
	for (int i = 0; i < 3; ++i)
	{
		const int c = 16 << i;
		n.pooled[i] = own(device_alloc<bf16>(voxels_at(n, i + 1) * c));
		n.grad_pooled[i] = own(device_alloc<bf16>(voxels_at(n, i + 1) * c));
		n.grad_skip[i] = own(device_alloc<bf16>(voxels_at(n, i) * c));
	}
	n.output = own(device_alloc<float>(voxels_at(n, 0)));
}

// He-normal weights from a seeded generator (the head at a hundredth of
// that, so the untrained network is close to the identity), zero biases.
void initialize(net_t &n, uint64_t seed)
{
	std::vector<float> host(static_cast<size_t>(n.parameter_count), 0.0f);
	std::mt19937_64 rng(seed);
	for (int l = 0; l < LAYERS; ++l)
	{
		const double sd = std::sqrt(2.0 / static_cast<double>(fan_in(defs[l]))) * (l == L_HEAD ? 0.01 : 1.0);
		std::normal_distribution<double> normal(0.0, sd);
		for (int64_t k = 0; k < weight_count(defs[l]); ++k)
			host[static_cast<size_t>(n.weight_offset[l] + k)] = static_cast<float>(normal(rng));
	}
	check_cuda(cudaMemcpy(n.params, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice),
		"upload of the prior's parameters");
}

// The BF16 copies and the flipped weights from the FP32 parameters.
void refresh(net_t &n, cudaStream_t stream)
{
	to_bf16_kernel<<<grid_for(n.parameter_count), 256, 0, stream>>>(n.parameter_count, n.params, n.params16);
	for (int l = 0; l < LAYERS; ++l)
		if (defs[l].kind == layer_kind::conv)
			flip_weights_kernel<<<grid_for(weight_count(defs[l])), 256, 0, stream>>>(n.params + n.weight_offset[l],
				defs[l].cout, defs[l].cin_a + defs[l].cin_b, n.flipped + n.flip_offset[l]);
	check_cuda(cudaGetLastError(), "refresh of the prior's weights");
}

// A 3x3x3 convolution through the tensor-core kernel.
void tc_conv(const net_t &n, int lvl, const bf16 *a, int ca, const bf16 *b, int cb, const bf16 *weights,
	const float *bias, int cout, int epilogue, bf16 *out0, int split, bf16 *out1, const bf16 *mask0, const bf16 *mask1,
	cudaStream_t stream)
{
	rexlib_b200_conv3d_args args{};
	args.sources = b != nullptr ? 2 : 1;
	args.inputs[0] = a;
	args.input_channels[0] = ca;
	args.input_strides[0] = ca;
	if (b != nullptr)
	{
		args.inputs[1] = b;
		args.input_channels[1] = cb;
		args.input_strides[1] = cb;
	}
	const int e = n.extent >> lvl;
	args.depth = args.height = args.width = e;
	args.weights = weights;
	args.bias = bias;
	args.output_channels = cout;
	args.epilogue = epilogue;
	args.outputs[0] = out0;
	args.output_strides[0] = split > 0 ? split : cout;
	args.output_split = split;
	if (split > 0)
	{
		args.outputs[1] = out1;
		args.output_strides[1] = cout - split;
	}
	args.masks[0] = mask0;
	args.masks[1] = mask1;
	args.mask_strides[0] = args.output_strides[0];
	args.mask_strides[1] = args.output_strides[1];
	args.error = n.error;
	const int32_t status = rexlib_b200_conv3d(&args, stream);
	if (status != REXLIB_B200_OK)
		fail(static_cast<rexlib_b200_status>(status), rexlib_b200_last_error());
}

} // anonymous namespace
} // namespace unet
} // namespace rexlib_b200

namespace rexlib_b200
{
namespace unet
{
namespace
{

const bf16 *weights16(const net_t &n, int l) { return n.params16 + n.weight_offset[l]; }
const float *bias32(const net_t &n, int l) { return n.params + n.bias_offset[l]; }

void forward(net_t &n, const float *input, float *output, cudaStream_t s)
{
	n.input = input;
	const volume_shape s0 = shape_at(n, 0);
	first_conv_kernel<<<grid_for(voxels_at(n, 0) / 2), 256, 0, s>>>(s0, input, n.params + n.weight_offset[L_FIRST],
		bias32(n, L_FIRST), n.act[L_FIRST]);
	auto conv = [&](int l, const bf16 *a, const bf16 *b) {
		const layer_def &d = defs[l];
		tc_conv(n, level_of(l), a, d.cin_a, b, d.cin_b, weights16(n, l), bias32(n, l), d.cout, 1, n.act[l], 0, nullptr,
			nullptr, nullptr, s);
	};
	auto pool = [&](int from, int i) {
		const volume_shape sh = shape_at(n, i);
		pool_kernel<<<grid_for(voxels_at(n, i + 1) * defs[from].cout / 8), 256, 0, s>>>(sh, defs[from].cout, n.act[from],
			n.pooled[i]);
	};
	auto up = [&](int l, const bf16 *x) {
		const layer_def &d = defs[l];
		const volume_shape sh = shape_at(n, level_of(l) + 1);
		// On the tensor cores: a GEMM over the input voxels with (sub-position,
		// output channel) columns, each written to its output voxel.
		conv3d_transposed2(x, d.cin_a, sh.d, sh.h, sh.w, weights16(n, l), bias32(n, l), d.cout, n.act[l], n.error, s);
	};
	conv(L_E0, n.act[L_FIRST], nullptr);
	pool(L_E0, 0);
	conv(L_E1A, n.pooled[0], nullptr);
	conv(L_E1, n.act[L_E1A], nullptr);
	pool(L_E1, 1);
	conv(L_E2A, n.pooled[1], nullptr);
	conv(L_E2, n.act[L_E2A], nullptr);
	pool(L_E2, 2);
	conv(L_B1, n.pooled[2], nullptr);
	conv(L_B2, n.act[L_B1], nullptr);
	up(L_UP2, n.act[L_B2]);
	conv(L_D2A, n.act[L_UP2], n.act[L_E2]);
	conv(L_D2, n.act[L_D2A], nullptr);
	up(L_UP1, n.act[L_D2]);
	conv(L_D1A, n.act[L_UP1], n.act[L_E1]);
	conv(L_D1, n.act[L_D1A], nullptr);
	up(L_UP0, n.act[L_D1]);
	conv(L_D0A, n.act[L_UP0], n.act[L_E0]);
	conv(L_D0, n.act[L_D0A], nullptr);
	head_kernel<<<grid_for(voxels_at(n, 0)), 256, 0, s>>>(voxels_at(n, 0), 16, n.act[L_D0],
		n.params + n.weight_offset[L_HEAD], bias32(n, L_HEAD), input, output);
	check_cuda(cudaGetLastError(), "prior forward");
	n.output = output;
}

// Gradients of 0.5 mean (y - target)^2 (added to the parameters' gradients;
// the loss added to *loss) after a forward pass.
void backward(net_t &n, const float *target, float *loss, cudaStream_t s)
{
	float *grad = n.grads;
	auto wgrad = [&](int l, const bf16 *a, const bf16 *b, const bf16 *g) {
		const layer_def &d = defs[l];
		const int lvl = level_of(l);
		const int cin = d.cin_a + d.cin_b;
		if ((n.extent >> lvl) >= 16)
		{
			// On the tensor cores: a GEMM over voxels with taps x input
			// channels as its rows.
			rexlib_b200_conv3d_wgrad_args w{};
			w.sources = b != nullptr ? 2 : 1;
			w.inputs[0] = a;
			w.input_channels[0] = w.input_strides[0] = d.cin_a;
			if (b != nullptr)
			{
				w.inputs[1] = b;
				w.input_channels[1] = w.input_strides[1] = d.cin_b;
			}
			w.depth = w.height = w.width = n.extent >> lvl;
			w.output_grad = g;
			w.output_channels = w.output_grad_stride = d.cout;
			w.weight_grad = grad + n.weight_offset[l];
			w.bias_grad = grad + n.bias_offset[l];
			w.error = n.error;
			const int32_t status = rexlib_b200_conv3d_wgrad(&w, s);
			if (status != REXLIB_B200_OK)
				fail(static_cast<rexlib_b200_status>(status), rexlib_b200_last_error());
			return;
		}
		// Levels narrower than 16 voxels: on the CUDA cores.
		const int cols = 4 * wgrad_threads / (d.cout / 4);
		const int splits = (27 * cin + cols - 1) / cols;
		const size_t smem = sizeof(float) * wgrad_chunk * (d.cout + cols);
		const int64_t v = voxels_at(n, lvl);
		// Voxel ranges of whole chunks, about six blocks an SM in all.
		const int64_t ranges = std::max<int64_t>(1, std::min<int64_t>((v + wgrad_chunk - 1) / wgrad_chunk,
			(148 * 6 + splits - 1) / splits));
		const int64_t per_block = ((v + ranges - 1) / ranges + wgrad_chunk - 1) / wgrad_chunk * wgrad_chunk;
		const dim3 grid(static_cast<unsigned>((v + per_block - 1) / per_block), static_cast<unsigned>(splits));
		auto run = [&](auto kernel) {
			kernel<<<grid, wgrad_threads, smem, s>>>(shape_at(n, lvl), a, d.cin_a, d.cin_a, b, d.cin_b, d.cin_b, g,
				grad + n.weight_offset[l], grad + n.bias_offset[l], per_block);
		};
		switch (d.cout)
		{
		case 16: run(wgrad_kernel<16>); break;
		case 32: run(wgrad_kernel<32>); break;
		case 64: run(wgrad_kernel<64>); break;
		default: run(wgrad_kernel<128>); break;
		}
	};
	// Input gradient of conv l: the convolution of its output gradient with
	// the flipped weights, masked by each input's ReLU where it had one.
	auto dgrad = [&](int l, bf16 *out0, bf16 *out1, const bf16 *mask0, const bf16 *mask1) {
		const layer_def &d = defs[l];
		const int cin = d.cin_a + d.cin_b;
		tc_conv(n, level_of(l), n.grad_a[l], d.cout, nullptr, 0, n.flipped + n.flip_offset[l], nullptr, cin,
			(mask0 || mask1) ? 2 : 0, out0, d.cin_b > 0 ? d.cin_a : 0, out1, mask0, mask1, s);
	};
	auto up_back = [&](int l, const bf16 *x, bf16 *dx) {
		const layer_def &d = defs[l];
		const volume_shape sh = shape_at(n, level_of(l) + 1);
		const int64_t v = voxels_at(n, level_of(l) + 1);
		// Weight gradient: a GEMM over the input's voxels with rows (sub-position,
		// output channel), about six blocks an SM over the column splits.
		const int rows = 8 * d.cout;
		const int cols = 4 * wgrad_threads / (rows / 4);
		const int splits = (d.cin_a + cols - 1) / cols;
		const int64_t ranges = std::max<int64_t>(1, std::min<int64_t>((v + wgrad_chunk - 1) / wgrad_chunk,
			(148 * 6 + splits - 1) / splits));
		const int64_t per_block = ((v + ranges - 1) / ranges + wgrad_chunk - 1) / wgrad_chunk * wgrad_chunk;
		const dim3 grid(static_cast<unsigned>((v + per_block - 1) / per_block), static_cast<unsigned>(splits));
		const size_t smem = sizeof(float) * wgrad_chunk * (rows + cols);
		auto run = [&](auto kernel) {
			kernel<<<grid, wgrad_threads, smem, s>>>(sh, x, d.cin_a, d.cin_a, nullptr, 0, 0, n.grad_a[l],
				grad + n.weight_offset[l], grad + n.bias_offset[l], per_block);
		};
		switch (rows)
		{
		case 128: run(wgrad_kernel<128, true>); break;
		case 256: run(wgrad_kernel<256, true>); break;
		default: run(wgrad_kernel<512, true>); break;
		}
		up_grad_input_kernel<<<dim3(grid_for(v), d.cin_a / 16), 256, sizeof(float) * 8 * 16 * d.cout, s>>>(sh, d.cin_a,
			d.cout, x,
			n.params + n.weight_offset[l], n.grad_a[l], dx);
	};
	auto skip_pool = [&](int l, int i) {
		const int c = defs[l].cout;
		skip_pool_grad_kernel<<<grid_for(voxels_at(n, i) * c / 8), 256, 0, s>>>(shape_at(n, i), c, n.act[l],
			n.grad_skip[i], n.grad_pooled[i], n.grad_a[l]);
	};
	head_loss_grad_kernel<<<grid_for(voxels_at(n, 0)), 256, 0, s>>>(voxels_at(n, 0), 16, n.act[L_D0],
		n.params + n.weight_offset[L_HEAD], n.output, target, n.grad_a[L_D0], grad + n.weight_offset[L_HEAD],
		grad + n.bias_offset[L_HEAD], loss);
	// Level 0 of the decoder.
	wgrad(L_D0, n.act[L_D0A], nullptr, n.grad_a[L_D0]);
	dgrad(L_D0, n.grad_a[L_D0A], nullptr, n.act[L_D0A], nullptr);
	wgrad(L_D0A, n.act[L_UP0], n.act[L_E0], n.grad_a[L_D0A]);
	dgrad(L_D0A, n.grad_a[L_UP0], n.grad_skip[0], nullptr, n.act[L_E0]);
	up_back(L_UP0, n.act[L_D1], n.grad_a[L_D1]);
	// Level 1.
	wgrad(L_D1, n.act[L_D1A], nullptr, n.grad_a[L_D1]);
	dgrad(L_D1, n.grad_a[L_D1A], nullptr, n.act[L_D1A], nullptr);
	wgrad(L_D1A, n.act[L_UP1], n.act[L_E1], n.grad_a[L_D1A]);
	dgrad(L_D1A, n.grad_a[L_UP1], n.grad_skip[1], nullptr, n.act[L_E1]);
	up_back(L_UP1, n.act[L_D2], n.grad_a[L_D2]);
	// Level 2.
	wgrad(L_D2, n.act[L_D2A], nullptr, n.grad_a[L_D2]);
	dgrad(L_D2, n.grad_a[L_D2A], nullptr, n.act[L_D2A], nullptr);
	wgrad(L_D2A, n.act[L_UP2], n.act[L_E2], n.grad_a[L_D2A]);
	dgrad(L_D2A, n.grad_a[L_UP2], n.grad_skip[2], nullptr, n.act[L_E2]);
	up_back(L_UP2, n.act[L_B2], n.grad_a[L_B2]);
	// Bottom.
	wgrad(L_B2, n.act[L_B1], nullptr, n.grad_a[L_B2]);
	dgrad(L_B2, n.grad_a[L_B1], nullptr, n.act[L_B1], nullptr);
	wgrad(L_B1, n.pooled[2], nullptr, n.grad_a[L_B1]);
	dgrad(L_B1, n.grad_pooled[2], nullptr, nullptr, nullptr);
	// Encoder.
	skip_pool(L_E2, 2);
	wgrad(L_E2, n.act[L_E2A], nullptr, n.grad_a[L_E2]);
	dgrad(L_E2, n.grad_a[L_E2A], nullptr, n.act[L_E2A], nullptr);
	wgrad(L_E2A, n.pooled[1], nullptr, n.grad_a[L_E2A]);
	dgrad(L_E2A, n.grad_pooled[1], nullptr, nullptr, nullptr);
	skip_pool(L_E1, 1);
	wgrad(L_E1, n.act[L_E1A], nullptr, n.grad_a[L_E1]);
	dgrad(L_E1, n.grad_a[L_E1A], nullptr, n.act[L_E1A], nullptr);
	wgrad(L_E1A, n.pooled[0], nullptr, n.grad_a[L_E1A]);
	dgrad(L_E1A, n.grad_pooled[0], nullptr, nullptr, nullptr);
	skip_pool(L_E0, 0);
	wgrad(L_E0, n.act[L_FIRST], nullptr, n.grad_a[L_E0]);
	dgrad(L_E0, n.grad_a[L_FIRST], nullptr, n.act[L_FIRST], nullptr);
	{
		// One block an SM (its registers take about half the SM's), fewer
		// for small volumes; each block's sums are added once.
		const int64_t chunks = (voxels_at(n, 0) + 63) / 64;
		const int blocks = static_cast<int>(std::min<int64_t>(chunks, 148));
		first_conv_grad_kernel<<<blocks, first_grad_threads, 0, s>>>(shape_at(n, 0), n.input, n.grad_a[L_FIRST],
			grad + n.weight_offset[L_FIRST], grad + n.bias_offset[L_FIRST]);
	}
	check_cuda(cudaGetLastError(), "prior backward");
}

void adam_step(net_t &n, float lr, cudaStream_t s)
{
	++n.steps;
	const float b1 = 1.0f - std::pow(0.9f, static_cast<float>(n.steps));
	const float b2 = 1.0f - std::pow(0.999f, static_cast<float>(n.steps));
	adam_kernel<<<grid_for(n.parameter_count), 256, 0, s>>>(n.parameter_count, n.params, n.grads, n.adam_m, n.adam_v,
		lr, b1, b2);
	check_cuda(cudaGetLastError(), "prior Adam step");
	refresh(n, s);
}

} // anonymous namespace
} // namespace unet
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_unet_create(int32_t extent, uint64_t seed, rexlib_b200_unet **net)
{
	return guarded([&] {
		require(net != nullptr, "null result pointer");
		*net = nullptr;
		if (extent < 16 || extent > 512 || (extent & (extent - 1)) != 0)
			fail(REXLIB_B200_UNSUPPORTED, "the prior takes cubic volumes of 16 to 512, a power of two");
		auto *n = new rexlib_b200_unet();
		n->extent = extent;
		try
		{
			unet::allocate(*n);
			unet::initialize(*n, seed);
			unet::refresh(*n, nullptr);
			check_cuda(cudaStreamSynchronize(nullptr), "prior set-up");
		}
		catch (...)
		{
			for (void *p : n->owned)
				cudaFree(p);
			delete n;
			throw;
		}
		*net = n;
	});
}

extern "C" int32_t rexlib_b200_unet_destroy(rexlib_b200_unet *net)
{
	return guarded([&] {
		if (net == nullptr)
			return;
		cudaDeviceSynchronize();
		for (void *p : net->owned)
			cudaFree(p);
		delete net;
	});
}

extern "C" int32_t rexlib_b200_unet_parameter_count(const rexlib_b200_unet *net, int64_t *count)
{
	return guarded([&] {
		require(net != nullptr && count != nullptr, "null network");
		*count = net->parameter_count;
	});
}

extern "C" int32_t rexlib_b200_unet_copy(rexlib_b200_unet *net, float *parameters_out, float *gradients_out,
	const float *parameters_in, void *stream)
{
	return guarded([&] {
		require(net != nullptr, "null network");
		const cudaStream_t s = as_stream(stream);
		const size_t bytes = sizeof(float) * static_cast<size_t>(net->parameter_count);
		if (parameters_out)
			check_cuda(cudaMemcpyAsync(parameters_out, net->params, bytes, cudaMemcpyDefault, s), "parameter copy");
		if (gradients_out)
			check_cuda(cudaMemcpyAsync(gradients_out, net->grads, bytes, cudaMemcpyDefault, s), "gradient copy");
		if (parameters_in)
		{
			check_cuda(cudaMemcpyAsync(net->params, parameters_in, bytes, cudaMemcpyDefault, s), "parameter copy");
			unet::refresh(*net, s);
		}
	});
}

extern "C" int32_t rexlib_b200_unet_tensor(rexlib_b200_unet *net, int32_t which, int32_t layer, void *out,
	void *stream)
{
	return guarded([&] {
		require(net != nullptr && out != nullptr && layer >= 0 && layer < unet::L_HEAD, "no such tensor");
		require(which == 0 || which == 1, "which: 0 for an activation, 1 for its gradient");
		const int64_t v = unet::voxels_at(*net, unet::level_of(layer));
		const size_t bytes = sizeof(__nv_bfloat16) * static_cast<size_t>(v) * unet::defs[layer].cout;
		check_cuda(cudaMemcpyAsync(out, which == 0 ? net->act[layer] : net->grad_a[layer], bytes, cudaMemcpyDefault,
					   as_stream(stream)),
			"tensor copy");
	});
}

extern "C" int32_t rexlib_b200_unet_layer(const rexlib_b200_unet *net, int32_t layer, int64_t *weight_offset,
	int64_t *bias_offset, int32_t *shape)
{
	return guarded([&] {
		require(net != nullptr && layer >= 0 && layer < unet::LAYERS, "no such layer");
		const auto &d = unet::defs[layer];
		*weight_offset = net->weight_offset[layer];
		*bias_offset = net->bias_offset[layer];
		shape[0] = static_cast<int32_t>(d.kind);
		shape[1] = d.cin_a;
		shape[2] = d.cin_b;
		shape[3] = d.cout;
	});
}

extern "C" int32_t rexlib_b200_unet_forward(rexlib_b200_unet *net, const float *input, float *output, void *stream)
{
	return guarded([&] {
		require(net != nullptr && input != nullptr && output != nullptr, "null network or volume");
		unet::forward(*net, input, output, as_stream(stream));
	});
}

extern "C" int32_t rexlib_b200_unet_backward(rexlib_b200_unet *net, const float *target, float *loss, void *stream)
{
	return guarded([&] {
		require(net != nullptr && target != nullptr && loss != nullptr, "null network, target or loss");
		require(net->input != nullptr, "backward needs a forward pass first");
		unet::backward(*net, target, loss, as_stream(stream));
	});
}

extern "C" int32_t rexlib_b200_unet_adam_step(rexlib_b200_unet *net, float learning_rate, void *stream)
{
	return guarded([&] {
		require(net != nullptr, "null network");
		unet::adam_step(*net, learning_rate, as_stream(stream));
	});
}

extern "C" int32_t rexlib_b200_unet_error(rexlib_b200_unet *net, int32_t *code)
{
	return guarded([&] {
		require(net != nullptr && code != nullptr, "null network");
		check_cuda(cudaMemcpy(code, net->error, sizeof(int32_t), cudaMemcpyDeviceToHost), "error word");
	});
}
