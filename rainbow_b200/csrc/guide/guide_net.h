// Learned path guiding: geometry of the network, its parameter layouts, and
// the guide density / sampler shared by the tensor-core kernels (guide.cu) and
// the path-continuation code of the wavefront shading kernels.
//
// Network: 9 inputs in [0, 1] -> 12-frequency sin/cos encoding (216 features,
// padded to 224) -> 4 hidden ReLU layers of width 64 -> 48 outputs: 8 vMF lobes
// (mean 3, log-concentration 1, weight logit 1) at 5 i .. 5 i + 4, the
// guide-vs-BSDF mixing logit at 40, 41..47 unused.
//
// On the device every bias is folded into its weight matrix as one more input
// column multiplied by a constant-1 feature: feature 216 of the encoded input
// (bias of layer 1), feature 64 of every hidden activation (bias of layers
// 2..5). Hidden activations are therefore stored 80 wide (64 values, the
// constant 1, 15 zeros) and every layer is one plain product on the tensor
// cores, forward and backward, with the bias gradient coming out of the
// weight-gradient product.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define RB_GHD __host__ __device__ __forceinline__
#else
#define RB_GHD inline
#endif

namespace rb {
namespace guide {

constexpr int kInputs = 9;
constexpr int kFreqs = 12;
constexpr int kFeatures = 216;        // kInputs * kFreqs * 2
constexpr int kK1 = 224;              // encoded input width (K of layer 1)
constexpr int kHidden = 64;
constexpr int kHiddenK = 80;          // stored hidden width (K of layers 2..5)
constexpr int kOutputs = 48;
constexpr int kLobes = 8;
constexpr int kLayers = 5;
constexpr int kBiasFeature1 = 216;    // constant-1 feature of the encoded input
constexpr int kNumParams = 30000;     // logical parameters, flat W1 b1 W2 b2 .. W5 b5
constexpr int kAugParams = 33536;     // device parameters, per layer [out][K] with the bias column
constexpr uint32_t kImageBytes = 2u * kAugParams;  // bf16 image of all layers (67,072 bytes)
constexpr int kTileRows = 128;        // rows per tensor-core tile (MMA M)

constexpr float kKappaMin = -4.f, kKappaMax = 8.f;   // clamp of the log-concentration
constexpr float kAlphaLo = 0.1f, kAlphaHi = 0.9f;    // range of the guide selection probability
constexpr float kEpsUniform = 0.02f;                 // uniform share of the guide density
constexpr float kNormFloor = 1e-6f;
constexpr float kPi = 3.14159265358979323846f;

RB_GHD int layer_out(int l) { return l == kLayers - 1 ? kOutputs : kHidden; }
RB_GHD int layer_in(int l) { return l == 0 ? kK1 : kHidden; }        // logical input width
RB_GHD int layer_k(int l) { return l == 0 ? kK1 : kHiddenK; }        // stored input width
RB_GHD int layer_bias_col(int l) { return l == 0 ? kBiasFeature1 : kHidden; }
// first device parameter of layer l ([out][K] row-major, bias in column layer_bias_col)
RB_GHD int aug_offset(int l) { return l == 0 ? 0 : kHidden * kK1 + (l - 1) * kHidden * kHiddenK; }
// first logical parameter of layer l (W [out][in] then b [out])
RB_GHD int flat_offset(int l) {
	return l == 0 ? 0 : (kHidden * kK1 + kHidden) + (l - 1) * (kHidden * kHidden + kHidden);
}

// Element offset of W_l[o][k] in the bf16 image: per layer, 8 x 8 core
// matrices [o / 8][k / 8][o % 8][k % 8] (the no-swizzle K-major operand layout
// with LBO = 128 bytes and SBO = K * 16 bytes; read MN-major for the backward
// product with LBO = K * 16 bytes and SBO = 128 bytes).
RB_GHD uint32_t image_index(int l, int o, int k) {
	const int K = layer_k(l);
	return static_cast<uint32_t>(aug_offset(l) + ((o >> 3) * (K >> 3) + (k >> 3)) * 64 + (o & 7) * 8 + (k & 7));
}

// Device parameter a -> (layer, out, k). Inverse of aug_offset + o * K + k.
RB_GHD void aug_coords(int a, int& l, int& o, int& k) {
	l = 0;
	while (l + 1 < kLayers && a >= aug_offset(l + 1)) l++;
	const int r = a - aug_offset(l);
	o = r / layer_k(l);
	k = r % layer_k(l);
}

// Logical parameter index of device parameter (l, o, k), or -1 for a padding
// column that has no logical counterpart (layer-1 columns 217..223, hidden
// columns 65..79). The bias column maps to b_l[o].
RB_GHD int aug_to_flat(int l, int o, int k) {
	const int in = layer_in(l), out = layer_out(l);
	if (k == layer_bias_col(l)) return flat_offset(l) + out * in + o;
	if (l == 0 ? (k >= kFeatures) : (k >= kHidden)) return -1;
	return flat_offset(l) + o * in + k;
}

// ------------------------------------------------------------ guide density
// Decoded guide of one query (48 floats, 12 float4): lobe i as (mu_i, kappa_i)
// at 4 i, the lobe's density factor (1 - eps) w_i c(kappa_i) at 32 + i, the
// cumulative lobe weights w_0 .. w_0 + .. + w_6 at 40 (the last lobe takes the
// rest of 1), alpha at 47.
constexpr int kLobeOff = 0, kWcOff = 32, kCdfOff = 40, kAlphaOff = 47;

RB_GHD float vmf_norm(float kappa) { return kappa / (2.f * kPi * (-expm1f(-2.f * kappa))); }

// q(d) = (1 - eps) sum_i w_i c(kappa_i) exp(kappa_i (mu_i . d - 1)) + eps / (4 pi)
RB_GHD float guide_pdf(const float* g, float dx, float dy, float dz) {
	const float4* g4 = reinterpret_cast<const float4*>(g);
	const float4 wa = g4[kWcOff / 4], wb = g4[kWcOff / 4 + 1];
	const float wc[kLobes] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
	float s = 0.f;
	for (int i = 0; i < kLobes; i++) {
		const float4 m = g4[kLobeOff / 4 + i];
		s += wc[i] * expf(m.w * ((m.x * dx + m.y * dy + m.z * dz) - 1.f));
	}
	return s + kEpsUniform / (4.f * kPi);
}

// Orthonormal basis (t, b) around unit n: Duff et al. 2017, "Building an
// Orthonormal Basis, Revisited".
RB_GHD void onb(float nx, float ny, float nz, float* t, float* b) {
	const float sign = nz >= 0.f ? 1.f : -1.f;
	const float a = -1.f / (sign + nz);
	const float bb = nx * ny * a;
	t[0] = 1.f + sign * nx * nx * a; t[1] = sign * bb; t[2] = -sign * nx;
	b[0] = bb; b[1] = sign + ny * ny * a; b[2] = -ny;
}

// Direction from q. u_pick < eps: uniform sphere (z = 1 - 2 u1, phi = 2 pi u2);
// otherwise (u_pick - eps) / (1 - eps) picks a lobe by cumulative weight and
// (u1, u2) sample it with Jakob's stable inversion (2012, "Numerically stable
// sampling of the von Mises-Fisher distribution on S^2"):
// cos = 1 + log(e^{-2 kappa} + u1 (1 - e^{-2 kappa})) / kappa.
RB_GHD void guide_sample(const float* g, float u_pick, float u1, float u2, float* d) {
	const float4* g4 = reinterpret_cast<const float4*>(g);
	float cz, m[3] = {0.f, 0.f, 1.f};
	if (u_pick < kEpsUniform) {
		cz = 1.f - 2.f * u1;
	} else {
		const float up = (u_pick - kEpsUniform) / (1.f - kEpsUniform);
		const float4 ca = g4[kCdfOff / 4], cb = g4[kCdfOff / 4 + 1];
		const float cdf[kLobes - 1] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z};
		int j = kLobes - 1;
		for (int i = 0; i < kLobes - 1; i++) {
			if (up < cdf[i]) { j = i; break; }
		}
		const float4 lb = g4[kLobeOff / 4 + j];
		const float k = lb.w;
		const float e2 = expf(-2.f * k);
		cz = 1.f + logf(e2 + u1 * (1.f - e2)) / k;
		m[0] = lb.x; m[1] = lb.y; m[2] = lb.z;
	}
	cz = fminf(1.f, fmaxf(-1.f, cz));
	const float s = sqrtf(fmaxf(0.f, 1.f - cz * cz));
	const float ph = 2.f * kPi * u2;
	const float cp = cosf(ph), sp = sinf(ph);
	float t[3], b[3];
	onb(m[0], m[1], m[2], t, b);
	for (int c = 0; c < 3; c++) d[c] = cz * m[c] + s * (cp * t[c] + sp * b[c]);
}

// Raw network outputs (48) -> decoded guide (48 floats, see kLobeOff ..).
RB_GHD void decode_outputs(const float* o, float* g) {
	float lmax = o[4];
	for (int i = 1; i < kLobes; i++) lmax = fmaxf(lmax, o[5 * i + 4]);
	float e[kLobes], esum = 0.f;
	for (int i = 0; i < kLobes; i++) { e[i] = expf(o[5 * i + 4] - lmax); esum += e[i]; }
	float acc = 0.f;
	for (int i = 0; i < kLobes; i++) {
		const float mx = o[5 * i], my = o[5 * i + 1], mz = o[5 * i + 2];
		const float nr = sqrtf(mx * mx + my * my + mz * mz);
		if (nr > 1e-12f) {
			g[kLobeOff + 4 * i] = mx / nr; g[kLobeOff + 4 * i + 1] = my / nr; g[kLobeOff + 4 * i + 2] = mz / nr;
		} else {
			g[kLobeOff + 4 * i] = 0.f; g[kLobeOff + 4 * i + 1] = 0.f; g[kLobeOff + 4 * i + 2] = 1.f;
		}
		const float k = expf(fminf(kKappaMax, fmaxf(kKappaMin, o[5 * i + 3])));
		const float w = e[i] / esum;
		g[kLobeOff + 4 * i + 3] = k;
		g[kWcOff + i] = (1.f - kEpsUniform) * w * vmf_norm(k);
		if (i < kLobes - 1) {
			acc += w;
			g[kCdfOff + i] = acc;
		}
	}
	g[kAlphaOff] = kAlphaLo + (kAlphaHi - kAlphaLo) / (1.f + expf(-o[40]));
}

// Gradient of the per-sample loss
//   -weight * (log q(d) + log(alpha q(d) + (1 - alpha) p_bsdf)) * inv_n
// with respect to the 48 raw outputs; returns the loss term.
RB_GHD float output_grad(const float* o, float dx, float dy, float dz, float weight, float p_bsdf, float inv_n, float* gout) {
	float lmax = o[4];
	for (int i = 1; i < kLobes; i++) lmax = fmaxf(lmax, o[5 * i + 4]);
	float w[kLobes], esum = 0.f;
	for (int i = 0; i < kLobes; i++) { w[i] = expf(o[5 * i + 4] - lmax); esum += w[i]; }
	float comp[kLobes], q = 0.f;
	for (int i = 0; i < kLobes; i++) {
		w[i] = w[i] / esum;
		const float mx = o[5 * i], my = o[5 * i + 1], mz = o[5 * i + 2];
		const float nr = sqrtf(mx * mx + my * my + mz * mz);
		float ux = 0.f, uy = 0.f, uz = 1.f;
		if (nr > 1e-12f) { ux = mx / nr; uy = my / nr; uz = mz / nr; }
		const float k = expf(fminf(kKappaMax, fmaxf(kKappaMin, o[5 * i + 3])));
		const float dt = ux * dx + uy * dy + uz * dz;
		comp[i] = vmf_norm(k) * expf(k * (dt - 1.f));
		q += w[i] * comp[i];
	}
	q = (1.f - kEpsUniform) * q + kEpsUniform / (4.f * kPi);
	const float sg = 1.f / (1.f + expf(-o[40]));
	const float alpha = kAlphaLo + (kAlphaHi - kAlphaLo) * sg;
	const float mix = alpha * q + (1.f - alpha) * p_bsdf;
	if (weight == 0.f) {
		for (int i = 0; i < kOutputs; i++) gout[i] = 0.f;
		return 0.f;
	}
	const float loss = -weight * (logf(q) + logf(mix)) * inv_n;
	const float g_q = -weight * (1.f / q + alpha / mix) * inv_n;
	const float g_alpha = -weight * ((q - p_bsdf) / mix) * inv_n;
	float gw_dot_w = 0.f;
	for (int i = 0; i < kLobes; i++) gw_dot_w += (1.f - kEpsUniform) * g_q * comp[i] * w[i];
	for (int i = 0; i < kLobes; i++) {
		const float mx = o[5 * i], my = o[5 * i + 1], mz = o[5 * i + 2];
		const float nr = sqrtf(mx * mx + my * my + mz * mz);
		float ux = 0.f, uy = 0.f, uz = 1.f;
		if (nr > 1e-12f) { ux = mx / nr; uy = my / nr; uz = mz / nr; }
		const float lk = o[5 * i + 3];
		const float k = expf(fminf(kKappaMax, fmaxf(kKappaMin, lk)));
		const float dt = ux * dx + uy * dy + uz * dz;
		const float g_comp = (1.f - kEpsUniform) * g_q * w[i];
		const float g_w = (1.f - kEpsUniform) * g_q * comp[i];
		gout[5 * i + 4] = w[i] * (g_w - gw_dot_w);
		const float em = -expm1f(-2.f * k);
		const float dlogc = 1.f / k - 2.f * expf(-2.f * k) / em;
		const float gc = g_comp * comp[i];
		gout[5 * i + 3] = (lk > kKappaMin && lk < kKappaMax) ? gc * (dlogc + (dt - 1.f)) * k : 0.f;
		const float s = gc * k;  // g_mu = s * d
		const float proj = s * dt; // (g_mu . mu)
		const float inv = 1.f / fmaxf(nr, kNormFloor);
		gout[5 * i] = (s * dx - proj * ux) * inv;
		gout[5 * i + 1] = (s * dy - proj * uy) * inv;
		gout[5 * i + 2] = (s * dz - proj * uz) * inv;
	}
	gout[40] = g_alpha * (kAlphaHi - kAlphaLo) * sg * (1.f - sg);
	for (int i = 41; i < kOutputs; i++) gout[i] = 0.f;
	return loss;
}

} // namespace guide
} // namespace rb
