// Host side of the library: the Model/Profile API of libprofit 1.9.3
// (model.h:55-421, profile.h:79-261, convolve.h:68-209) over device buffers,
// and the C ABI declared in include/profit_b200.h.
//
// Evaluation mirrors Model::evaluate (model.cpp:271-338) and
// Model::produce_image (model.cpp:340-380): profiles marked `convolve` are
// drawn into one padded image, the others into a second one; the first is
// convolved with the normalised PSF, the PSF padding is cropped, the second
// is added, and finesampled images are summed back down when requested.
#include <algorithm>
#include <array>
#include <cctype>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <string>
#include <vector>

#include "conv.cuh"
#include "fft.h"
#include "launch.h"
#include "profit_b200.h"

using namespace pf;

namespace pf {
static std::atomic<unsigned long long> g_launches{0};
void note_launches(int n) { g_launches += (unsigned long long)n; }

cudaError_t conv_autotuned(const ConvCandidate *cands, int n_cands, int type_tag, const ConvArgs &a, cudaStream_t s)
{
	using Key = std::tuple<int, int, int, int, int, int, int, int>;
	static std::mutex mu;
	static std::map<Key, int> choice;
	Key key{type_tag, a.sw, a.sh, a.kw, a.kh, a.ow, a.oh, a.batch};
	// PF_CONV_FORCE=<index> runs that candidate whenever it applies (tests
	// check every candidate against the FP64 form this way)
	if (const char *fv = getenv("PF_CONV_FORCE")) {
		int f = fv[0] ? atoi(fv) : -1;
		if (f >= 0 && f < n_cands && cands[f].smem(a.kw, a.kh) <= 227 * 1024) {
			cudaError_t e = cands[f].run(a, s);
			if (e != cudaErrorInvalidValue) return e;
			cudaGetLastError();  // not applicable here: use the tuned choice
		}
	}
	int pick = -1;
	{
		std::lock_guard<std::mutex> g(mu);
		auto it = choice.find(key);
		if (it != choice.end()) pick = it->second;
	}
	if (pick < 0) {
		// A shape close to one already tuned (same direction, kernel sides in
		// the same 8-pixel class, the same power of two in output width and
		// in total output pixels) takes that choice: a catalogue brings
		// hundreds of chunk shapes that differ in canvas side, PSF size and
		// galaxy count, and timing every candidate for each one made its
		// first call last seconds.
		auto lg2 = [](long long v) {
			int r = 0;
			while (v > 1) {
				v >>= 1;
				r++;
			}
			return r;
		};
		const int wc = lg2(a.ow), nc = lg2((long long)a.ow * a.oh * a.batch);
		int near = -1;
		{
			std::lock_guard<std::mutex> g(mu);
			for (const auto &kv : choice) {
				const Key &k = kv.first;
				if (std::get<0>(k) == type_tag && std::get<3>(k) / 8 == a.kw / 8 && std::get<4>(k) / 8 == a.kh / 8 &&
				    lg2(std::get<5>(k)) == wc &&
				    lg2((long long)std::get<5>(k) * std::get<6>(k) * std::get<7>(k)) == nc) {
					near = kv.second;
					break;
				}
			}
		}
		if (near >= 0 && cands[near].smem(a.kw, a.kh) <= 227 * 1024) {
			cudaError_t e = cands[near].run(a, s);
			if (e != cudaErrorInvalidValue) {
				if (e == cudaSuccess) {
					std::lock_guard<std::mutex> g(mu);
					choice[key] = near;
				}
				return e;
			}
			cudaGetLastError();  // not applicable to this shape (scratch): tune it
		}
	}
	if (pick < 0) {
		cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
		cudaStreamIsCapturing(s, &cap);
		int first_fit = -1;
		for (int c = 0; c < n_cands; c++)
			if (cands[c].tuned && cands[c].smem(a.kw, a.kh) <= 227 * 1024) {
				first_fit = c;
				break;
			}
		if (first_fit < 0) return cudaErrorInvalidValue;
		if (cap != cudaStreamCaptureStatusNone) {
			pick = first_fit;  // no timing inside a capture
		}
		else {
			cudaEvent_t e0, e1;
			cudaEventCreate(&e0);
			cudaEventCreate(&e1);
			// PF_AUTOTUNE_LOG=1 prints every candidate's time to stderr
			const char *lv = getenv("PF_AUTOTUNE_LOG");
			const bool log = lv && lv[0] == '1';
			// Candidates are timed on the first images of a large batch only:
			// every candidate on about 512k output pixels, then the six
			// fastest again on about 2M (enough to fill every SM several
			// times over), the best of three runs each.  The ranking is per tile, and timing whole
			// catalogue chunks made the tuning most of a catalogue's first
			// call.  The runs write only outputs that the chosen candidate
			// then rewrites.
			const long long per = std::max(1LL, (long long)a.ow * a.oh);
			auto truncated = [&](long long pixels) {
				ConvArgs t = a;
				t.batch = (int)std::min<long long>(a.batch, std::max(1LL, (pixels + per - 1) / per));
				// scratch in proportion, so that a candidate needing it applies
				// to the truncated batch exactly when it applies to the whole one
				t.scratch_bytes = a.scratch_bytes / std::max(1, a.batch) * t.batch;
				return t;
			};
			auto time_one = [&](const ConvArgs &t, int c, bool warm, float &ms, int min_reps) -> bool {
				if (warm) {
					cudaError_t e = cands[c].run(t, s);  // warm-up (and attribute setup)
					if (e != cudaSuccess) {
						cudaGetLastError();
						return false;
					}
				}
				// batched shapes run long enough to be timed once per repetition;
				// the fastest repetition counts
				const int reps = std::max(min_reps, t.batch > 8 ? 1 : 3);
				ms = 1e30f;
				for (int r = 0; r < reps; r++) {
					cudaEventRecord(e0, s);
					cands[c].run(t, s);
					cudaEventRecord(e1, s);
					if (cudaEventSynchronize(e1) != cudaSuccess) return false;
					float one = 0;
					cudaEventElapsedTime(&one, e0, e1);
					ms = std::min(ms, one);
				}
				if (log)
					fprintf(stderr, "[profit_b200 autotune] type %d src %dx%d psf %dx%d out %dx%d batch %d (timed on %d): "
					        "candidate %d %.4f ms\n",
					        type_tag, a.sw, a.sh, a.kw, a.kh, a.ow, a.oh, a.batch, t.batch, c, ms);
				return true;
			};
			auto by_time = [](std::vector<std::pair<float, int>> &v) {
				std::stable_sort(v.begin(), v.end(), [](const std::pair<float, int> &x, const std::pair<float, int> &y) {
					return x.first < y.first;
				});
			};
			const ConvArgs t1 = truncated(1LL << 19), t2 = truncated(1LL << 21);
			std::vector<std::pair<float, int>> ranked;
			for (int c = 0; c < n_cands; c++) {
				if (!cands[c].tuned || cands[c].smem(a.kw, a.kh) > 227 * 1024) continue;
				float ms = 0;
				if (time_one(t1, c, true, ms, 1)) ranked.emplace_back(ms, c);
			}
			by_time(ranked);
			if (t2.batch > t1.batch) {
				const size_t top = std::min<size_t>(6, ranked.size());
				for (size_t r = 0; r < top; r++) time_one(t2, ranked[r].second, false, ranked[r].first, 3);
				std::vector<std::pair<float, int>> head(ranked.begin(), ranked.begin() + top);
				by_time(head);
				std::copy(head.begin(), head.end(), ranked.begin());
			}
			cudaEventDestroy(e0);
			cudaEventDestroy(e1);
			ranked.emplace_back(0.0f, first_fit);
			// the fastest that also takes the whole batch
			for (const auto &r : ranked) {
				cudaError_t e = cands[r.second].run(a, s);
				if (e == cudaErrorInvalidValue) {
					cudaGetLastError();
					continue;
				}
				if (log) fprintf(stderr, "[profit_b200 autotune] type %d: picked candidate %d\n", type_tag, r.second);
				if (e == cudaSuccess) {
					std::lock_guard<std::mutex> g(mu);
					choice[key] = r.second;
				}
				return e;
			}
			return cudaErrorInvalidValue;
		}
	}
	return cands[pick].run(a, s);
}
}  // namespace pf

namespace {

thread_local std::string g_error;

int set_error(int code, const std::string &msg)
{
	g_error = msg;
	return code;
}

#define PF_CUDA(...)                                                                                  \
	do {                                                                                              \
		cudaError_t e_ = (__VA_ARGS__);                                                               \
		if (e_ != cudaSuccess)                                                                        \
			return set_error(PF_E_CUDA, std::string(#__VA_ARGS__) + ": " + cudaGetErrorString(e_)); \
	} while (0)

// Timing events must become graph nodes when the stream is being captured
// (a plain record there only orders work); outside a capture the external
// flag is not allowed.
cudaError_t record_event(cudaEvent_t e, cudaStream_t s)
{
	cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
	cudaStreamIsCapturing(s, &st);
	if (st == cudaStreamCaptureStatusActive) return cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
	return cudaEventRecord(e, s);
}

#define PF_TRY(expr)          \
	do {                      \
		int st_ = (expr);     \
		if (st_ != PF_OK)     \
			return st_;       \
	} while (0)

struct DevBuf {
	void *p = nullptr;
	size_t bytes = 0;
	~DevBuf()
	{
		if (p) cudaFree(p);
	}
	template <class T>
	T *as() const
	{
		return static_cast<T *>(p);
	}
};

struct HostBuf {
	void *p = nullptr;
	size_t bytes = 0;
	~HostBuf()
	{
		if (p) cudaFreeHost(p);
	}
	template <class T>
	T *as() const
	{
		return static_cast<T *>(p);
	}
};

cudaError_t ensure(DevBuf &b, size_t bytes)
{
	if (bytes <= b.bytes && b.p) return cudaSuccess;
	if (b.p) cudaFree(b.p);
	b.p = nullptr;
	b.bytes = 0;
	size_t want = std::max<size_t>(bytes + bytes / 4, 256);
	cudaError_t e = cudaMalloc(&b.p, want);
	if (e == cudaSuccess) b.bytes = want;
	return e;
}

cudaError_t ensure(HostBuf &b, size_t bytes)
{
	if (bytes <= b.bytes && b.p) return cudaSuccess;
	if (b.p) cudaFreeHost(b.p);
	b.p = nullptr;
	b.bytes = 0;
	size_t want = std::max<size_t>(bytes + bytes / 4, 256);
	cudaError_t e = cudaMallocHost(&b.p, want);
	if (e == cudaSuccess) b.bytes = want;
	return e;
}

// Parameter registry: libprofit's register_parameter calls per profile.
enum PType { T_DOUBLE, T_UINT, T_BOOL };
struct ParamDesc {
	const char *name;
	PType type;
	size_t off;
};
#define PDD(n) {#n, T_DOUBLE, offsetof(ProfileParams, n)}
#define PDU(n) {#n, T_UINT, offsetof(ProfileParams, n)}
#define PDB(n) {#n, T_BOOL, offsetof(ProfileParams, n)}
const ParamDesc kRadial[] = {PDD(xcen), PDD(ycen), PDD(mag), PDD(ang), PDD(axrat), PDD(box), PDB(rough), PDB(adjust),
                             PDB(force_cpu), PDD(acc), PDD(rscale_switch), PDD(rscale_max), PDU(max_recursions),
                             PDU(resolution), PDB(convolve), {nullptr, T_DOUBLE, 0}};
const ParamDesc kSersic[] = {PDD(re), PDD(nser), PDB(rescale_flux), {nullptr, T_DOUBLE, 0}};
const ParamDesc kMoffat[] = {PDD(fwhm), PDD(con), {nullptr, T_DOUBLE, 0}};
const ParamDesc kFerrer[] = {PDD(rout), PDD(a), PDD(b), {nullptr, T_DOUBLE, 0}};
const ParamDesc kCoreSersic[] = {PDD(re), PDD(rb), PDD(nser), PDD(a), PDD(b), {nullptr, T_DOUBLE, 0}};
const ParamDesc kKing[] = {PDD(rc), PDD(rt), PDD(a), {nullptr, T_DOUBLE, 0}};
const ParamDesc kBrokenExp[] = {PDD(h1), PDD(h2), PDD(rb), PDD(a), {nullptr, T_DOUBLE, 0}};
const ParamDesc kSky[] = {PDD(bg), PDB(convolve), {nullptr, T_DOUBLE, 0}};
const ParamDesc kPsf[] = {PDD(xcen), PDD(ycen), PDD(mag), PDB(convolve), {nullptr, T_DOUBLE, 0}};
const ParamDesc kNull[] = {PDB(convolve), {nullptr, T_DOUBLE, 0}};

const char *kind_name(int k)
{
	static const char *names[] = {"sersic", "moffat", "ferrer", "coresersic", "king", "brokenexp", "sky", "psf", "null"};
	return (k >= 0 && k <= 8) ? names[k] : "?";
}

const ParamDesc *find_param(int kind, const char *name)
{
	const ParamDesc *lists[2] = {nullptr, nullptr};
	switch (kind) {
	case PK_SERSIC: lists[0] = kRadial; lists[1] = kSersic; break;
	case PK_MOFFAT: lists[0] = kRadial; lists[1] = kMoffat; break;
	case PK_FERRER: lists[0] = kRadial; lists[1] = kFerrer; break;
	case PK_CORESERSIC: lists[0] = kRadial; lists[1] = kCoreSersic; break;
	case PK_KING: lists[0] = kRadial; lists[1] = kKing; break;
	case PK_BROKENEXP: lists[0] = kRadial; lists[1] = kBrokenExp; break;
	case PK_SKY: lists[0] = kSky; break;
	case PK_PSF: lists[0] = kPsf; break;
	default: lists[0] = kNull; break;
	}
	for (auto *l : lists) {
		if (!l) continue;
		for (const ParamDesc *d = l; d->name; d++)
			if (std::strcmp(d->name, name) == 0) return d;
	}
	return nullptr;
}

ProfileParams default_params(int kind)
{
	ProfileParams p;
	std::memset(&p, 0, sizeof(p));
	p.kind = kind;
	// radial.cpp:724-752
	p.mag = 15;
	p.axrat = 1;
	p.acc = 0.1;
	p.rscale_switch = 1;
	p.resolution = 9;
	p.max_recursions = 2;
	p.adjust = 1;
	switch (kind) {
	case PK_SERSIC: p.re = 1; p.nser = 1; break;                              // sersic.cpp:350-359
	case PK_MOFFAT: p.fwhm = 3; p.con = 2; break;                             // moffat.cpp:102-108
	case PK_FERRER: p.rout = 3; p.a = 1; p.b = 1; p.acc = 1; break;           // ferrer.cpp:115-126
	case PK_CORESERSIC: p.re = 1; p.rb = 1; p.nser = 4; p.a = 1; p.b = 1; break;  // coresersic.cpp:131-140
	case PK_KING: p.rc = 1; p.rt = 3; p.a = 2; break;                         // king.cpp:111-119
	case PK_BROKENEXP: p.h1 = 1; p.h2 = 1; p.rb = 1; p.a = 1; break;          // brokenexponential.cpp:141-150
	case PK_PSF: p.mag = 0; break;                                            // psf.cpp:147-156
	default: break;
	}
	return p;
}

int kind_from_name(const char *name)
{
	// model.cpp:103-135
	if (!std::strcmp(name, "null")) return PK_NULL;
	if (!std::strcmp(name, "sky")) return PK_SKY;
	if (!std::strcmp(name, "sersic")) return PK_SERSIC;
	if (!std::strcmp(name, "moffat")) return PK_MOFFAT;
	if (!std::strcmp(name, "ferrer") || !std::strcmp(name, "ferrers")) return PK_FERRER;
	if (!std::strcmp(name, "coresersic")) return PK_CORESERSIC;
	if (!std::strcmp(name, "king")) return PK_KING;
	if (!std::strcmp(name, "brokenexp")) return PK_BROKENEXP;
	if (!std::strcmp(name, "psf")) return PK_PSF;
	return -1;
}

enum ConvKind { CONV_BRUTE = 0, CONV_FFT = 1, CONV_NULL = 2 };

struct Analysis {
	bool conv;
	unsigned padx, pady, dw, dh;  // drawing dims
	unsigned cw, ch;              // cropped dims (finesampled)
	unsigned ow, oh;              // output dims
	int levels;
	int n_profiles;
	// calculation mask (Model::analyze_expansion_requirements, model.cpp:152-183)
	bool mask = false;          // a drawing-size mask is in effect
	bool mask_adjusted = false; // it was built from the user's mask (adjust_mask)
	bool mask_conv = false;     // the convolution is masked by it
	bool mask_psf_pad = false;  // the user's mask needed the PSF padding
};

// Per-evaluation device results: [0] logL, [1..] tangent reductions.
struct ResultLayout {
	static constexpr int LL = 0;
	static constexpr int T0 = 8;
};

}  // namespace

struct BatchState;

struct pf_model {
	// per profile: its shape-only scalars, kept while nser and box are unchanged
	std::vector<pf::ShapeMemo> nq;
	unsigned width, height;
	std::vector<ProfileParams> profiles;
	std::vector<double> psf;  // normalised
	unsigned psf_w = 0, psf_h = 0;
	bool psf_dirty = true;
	double magzero = 0, sx = 1, sy = 1, psf_sx = 1, psf_sy = 1;
	unsigned fs = 1;
	bool return_fine = true, crop = true, debug = false;
	int conv_kind = CONV_BRUTE;
	int precision = PF_FP64;
	int device = 0;
	cudaStream_t stream = nullptr;
	cudaEvent_t ev[5] = {};
	float timings[4] = {0, 0, 0, 0};
	bool timings_lazy = false;  // timings still to be read from ev[] (FP32 pipeline)

	// device buffers
	DevBuf d_prof, d_fprof, d_prof_begin, d_prof_batch;
	DevBuf d_conv64, d_plain64, d_model64;
	DevBuf d_conv32, d_plain32, d_model32, d_jac, d_gconv, d_gplain, d_wseed;
	DevBuf d_psf64, d_psfrev64, d_psf32, d_psfrev32;
	DevBuf d_convsplit;  // FP64 partial images of column-split convolutions
	DevBuf d_jac_partials, d_jac_tickets;  // per-block sums and tickets of the tangent reduction
	DevBuf d_like_tickets;  // per-image tickets of the one-launch norm likelihood
	DevBuf d_items, d_masks, d_ctrl, d_partials, d_results;
	int adjoint_mode = PF_ADJOINT_AUTO;
	DevBuf d_decisions, d_level_counts;
	DevBuf d_data, d_sigma, d_region;
	// calculation mask (Model::set_mask / set_adjust_mask, model.h:196-214)
	std::vector<uint8_t> mask;
	unsigned mask_w = 0, mask_h = 0;
	bool adjust_mask = true;
	bool dry_run = false;
	std::vector<uint64_t> mask_key;  // what the device masks were built for
	uint64_t mask_version = 0;       // bumped by pf_model_set_mask
	DevBuf d_model_fine, d_seed_fine;  // FP32 pipeline: convolved fine image, fine seed
	DevBuf d_perm;                     // level items grouped by profile kind (QueueSet::perm)
	DevBuf d_mask_draw, d_mask_out;
	int like_kind = LIKE_NORM;
	DevBuf d_likestats;
	HostBuf h_prof, h_fprof, h_results, h_ctrl;
	std::vector<uint32_t> caps;
	bool has_data = false, has_region = false;
	unsigned data_w = 0, data_h = 0;

	// "fft" convolver: transforms, PSF spectra and work spectra
	FftConv<double> fft64;
	FftConv<float> fft32;
	DevBuf d_kspec64, d_kspec32, d_fftwork64, d_fftwork32;
	unsigned psf_version = 1, kspec64_version = 0, kspec32_version = 0;

	// captured FP32 likelihood+gradient pipeline (replayed while its signature holds)
	cudaGraphExec_t graph_exec = nullptr;
	std::vector<uint64_t> graph_sig;
	unsigned long long graph_kernels = 0;
	bool use_graphs = true;
	// phase events (render / convolution / likelihood and adjoint) inside
	// replayed graphs: off by default, since each event node costs the graph
	// microseconds; the total is timed by events around the launch
	bool phase_timing = false;
	bool phases_recorded = false;  // the last FP32 run recorded ev[1] and ev[2]
	int prof_begin_n = -1;
	BatchState *batch = nullptr;

	// fit space (pf_model_set_fit_space): the entries, the gradient
	// references of their free and tied entries, and the entries' device copy
	std::vector<FitEntry> fit_entries;
	std::vector<std::pair<int, std::string>> fit_refs;
	FitOffset fit_off{0.0, 0.0, 0.0, 1.0};
	int fit_nfit = 0;
	DevBuf d_fit_entries;
	uint64_t fit_version = 0;

	// debug output of the last evaluation
	std::vector<int32_t> decisions;
	std::vector<unsigned long long> level_counts;
	std::vector<unsigned long long> evals;  // [n_profiles][1 + MAX_LEVELS]
	unsigned dec_npix = 0;
	int dec_levels = 0;
};

namespace {

constexpr int NPARTS = LIKE_MAX_PARTS;  // likelihood partial sums (like_parts, common.cuh)
constexpr size_t CTRL_WORDS = 64;  // counts[16], overflow, ...

int analyze(pf_model *m, Analysis &a)
{
	if (m->width == 0 || m->height == 0) return set_error(PF_E_INVALID, "Model's requested dimensions are 0");
	if (m->sx <= 0) return set_error(PF_E_INVALID, "Model's scale_x cannot be negative or zero");
	if (m->sy <= 0) return set_error(PF_E_INVALID, "Model's scale_y cannot be negative or zero");
	if (m->profiles.empty()) return set_error(PF_E_INVALID, "No profiles provided in the model");
	a.conv = false;
	for (auto &p : m->profiles)
		if (p.convolve) a.conv = true;
	if (a.conv && m->psf.empty()) return set_error(PF_E_INVALID, "No psf provided but profile(s) requested convolution");
	a.levels = 1;
	for (auto &p : m->profiles) {
		const char *err = validate_profile(p, !m->psf.empty());
		if (err) return set_error(PF_E_INVALID, err);
		if (is_radial_kind(p.kind)) {
			// With adjust the resolution is derived in [4, 16] (radial.cpp:169-172);
			// otherwise the user's value is used as is.
			if (!p.adjust && !p.rough && (p.resolution == 0 || p.resolution > 16))
				return set_error(PF_E_INVALID, "resolution must be in [1, 16] when adjust is false");
			unsigned mr = p.max_recursions;
			if (p.kind == PK_SERSIC && p.adjust && p.nser > 1) mr = std::max(mr, 10u);
			if (mr + 1 > (unsigned)MAX_LEVELS)
				return set_error(PF_E_INVALID, "max_recursions above 15 is not supported");
			a.levels = std::max(a.levels, (int)mr + 1);
		}
	}
	if (m->profiles.size() > 65535) return set_error(PF_E_INVALID, "too many profiles");
	const bool has_mask = !m->mask.empty();
	if (has_mask && m->adjust_mask && (m->mask_w != m->width || m->mask_h != m->height))
		return set_error(PF_E_INVALID, "Mask dimensions != model dimensions");
	bool pad = a.conv;
	a.mask = has_mask;
	a.mask_adjusted = a.mask_conv = a.mask_psf_pad = false;
	if (has_mask && !m->adjust_mask) {
		// the mask is given at drawing size: padding iff it is larger than the image
		pad = m->mask_w > m->width * m->fs && m->mask_h > m->height * m->fs;
	}
	else if (has_mask && a.conv) {
		// no padding when the mask keeps psf/2 pixels clear of every edge
		unsigned lbx = m->mask_w, lby = m->mask_h, ubx = 0, uby = 0;
		bool any = false;
		for (unsigned j = 0; j < m->mask_h; j++)
			for (unsigned i = 0; i < m->mask_w; i++)
				if (m->mask[i + (size_t)j * m->mask_w]) {
					lbx = std::min(lbx, i);
					lby = std::min(lby, j);
					ubx = std::max(ubx, i + 1);
					uby = std::max(uby, j + 1);
					any = true;
				}
		if (!any) lbx = lby = ubx = uby = 0;
		const unsigned fs = m->fs, nx = m->psf_w / 2, ny = m->psf_h / 2;
		const unsigned low_x = lbx * fs, low_y = lby * fs;
		const unsigned up_x = m->mask_w * fs - ubx * fs, up_y = m->mask_h * fs - uby * fs;
		pad = !(low_x >= nx && low_y >= ny) || !(up_x >= nx && up_y >= ny);
		a.mask_conv = true;
		a.mask_psf_pad = pad;
	}
	if (has_mask && m->adjust_mask) a.mask_adjusted = a.mask_conv || a.mask_psf_pad || m->fs > 1;
	a.padx = pad ? m->psf_w / 2 : 0;
	a.pady = pad ? m->psf_h / 2 : 0;
	a.cw = m->width * m->fs;
	a.ch = m->height * m->fs;
	a.dw = a.cw + 2 * a.padx;
	a.dh = a.ch + 2 * a.pady;
	if ((size_t)a.dw * a.dh >= (1ull << 31)) return set_error(PF_E_INVALID, "image too large");
	if (m->fs > 1 && !m->return_fine) {
		a.ow = (a.cw + m->fs - 1) / m->fs;
		a.oh = (a.ch + m->fs - 1) / m->fs;
	}
	else {
		a.ow = a.cw;
		a.oh = a.ch;
	}
	a.n_profiles = (int)m->profiles.size();
	// crop = false (Model::evaluate, model.cpp:307-322) changes the result
	// only through the convolver's own padding: the brute-force and null
	// convolvers add none (Convolver::padding, convolve.cpp:50-53), so their
	// uncropped image is the cropped one.  The FFT convolver returns its whole
	// 2 max(src, psf) buffer (convolve.cpp:81-95, 263-268); that form is not
	// provided.
	if (!m->crop && a.conv && m->conv_kind == CONV_FFT)
		return set_error(PF_E_INVALID,
		                 "crop = false is supported with the brute, brute-old and null convolvers, not with fft");
	if (has_mask && !m->adjust_mask && (m->mask_w != a.dw || m->mask_h != a.dh))
		return set_error(PF_E_INVALID, "Mask dimensions != drawing dimensions: " + std::to_string(m->mask_w) + "x" +
		                                   std::to_string(m->mask_h) + " != " + std::to_string(a.dw) + "x" +
		                                   std::to_string(a.dh));
	return PF_OK;
}

// The drawing-size mask the profiles and the convolver see (Model::adjust,
// model.cpp:230-246): the user's mask upsampled by the finesampling factor,
// placed inside the PSF padding, and dilated by psf/2 pixels when the
// convolution is masked (Mask::expand_by, image.cpp:113-157, a box dilation,
// done here as a row pass then a column pass).  Without adjust_mask the
// user's mask is used as it is.  Also uploads the user's mask for the final
// image &= mask.  Rebuilt only when its inputs change.
int upload_masks(pf_model *m, const Analysis &a)
{
	if (!a.mask) return PF_OK;
	std::vector<uint64_t> key = {m->mask_w, m->mask_h, m->adjust_mask, m->fs,  m->psf_w,
	                             m->psf_h,  a.dw,      a.dh,           a.mask_conv, a.mask_psf_pad,
	                             m->mask_version};
	if (key == m->mask_key && m->d_mask_draw.p) return PF_OK;
	std::vector<uint8_t> draw;
	if (!m->adjust_mask) {
		draw = m->mask;
	}
	else {
		const unsigned fs = m->fs;
		draw.assign((size_t)a.dw * a.dh, 0);
		for (unsigned j = 0; j < m->mask_h * fs; j++)
			for (unsigned i = 0; i < m->mask_w * fs; i++)
				draw[(i + a.padx) + (size_t)(j + a.pady) * a.dw] = m->mask[i / fs + (size_t)(j / fs) * m->mask_w] ? 1 : 0;
		if (a.mask_conv) {
			const unsigned px = m->psf_w / 2, py = m->psf_h / 2;
			std::vector<uint8_t> rows(draw.size(), 0);
			for (unsigned j = 0; j < a.dh; j++) {
				const uint8_t *in = &draw[(size_t)j * a.dw];
				uint8_t *out = &rows[(size_t)j * a.dw];
				int last = -1;  // last set column seen so far
				std::vector<int> next(a.dw + 1, -1);
				int nx = -1;
				for (int i = (int)a.dw - 1; i >= 0; i--) {
					if (in[i]) nx = i;
					next[i] = nx;
				}
				for (unsigned i = 0; i < a.dw; i++) {
					if (in[i]) last = (int)i;
					bool hit = (last >= 0 && (int)i - last <= (int)px) || (next[i] >= 0 && next[i] - (int)i <= (int)px);
					out[i] = hit;
				}
			}
			for (unsigned i = 0; i < a.dw; i++) {
				int last = -1;
				std::vector<int> next(a.dh + 1, -1);
				int ny = -1;
				for (int j = (int)a.dh - 1; j >= 0; j--) {
					if (rows[i + (size_t)j * a.dw]) ny = j;
					next[j] = ny;
				}
				for (unsigned j = 0; j < a.dh; j++) {
					if (rows[i + (size_t)j * a.dw]) last = (int)j;
					bool hit = (last >= 0 && (int)j - last <= (int)py) || (next[j] >= 0 && next[j] - (int)j <= (int)py);
					draw[i + (size_t)j * a.dw] = hit;
				}
			}
		}
	}
	PF_CUDA(ensure(m->d_mask_draw, draw.size()));
	PF_CUDA(cudaMemcpy(m->d_mask_draw.p, draw.data(), draw.size(), cudaMemcpyHostToDevice));
	PF_CUDA(ensure(m->d_mask_out, m->mask.size()));
	PF_CUDA(cudaMemcpy(m->d_mask_out.p, m->mask.data(), m->mask.size(), cudaMemcpyHostToDevice));
	m->mask_key = key;
	return PF_OK;
}

ModelGeom geometry(const pf_model *m, const Analysis &a)
{
	ModelGeom g;
	g.magzero = m->magzero;
	g.sx = m->sx / m->fs;
	g.sy = m->sy / m->fs;
	g.img_sx = m->sx;
	g.img_sy = m->sy;
	g.offx = a.padx;
	g.offy = a.pady;
	g.finesampling = m->fs;
	return g;
}

int upload_psf(pf_model *m)
{
	if (!m->psf_dirty) return PF_OK;
	size_t n = m->psf.size();
	if (n == 0) {
		m->psf_dirty = false;
		return PF_OK;
	}
	std::vector<double> rev(m->psf.rbegin(), m->psf.rend());
	std::vector<float> f32(m->psf.begin(), m->psf.end()), r32(rev.begin(), rev.end());
	PF_CUDA(ensure(m->d_psf64, n * 8));
	PF_CUDA(ensure(m->d_psfrev64, n * 8));
	PF_CUDA(ensure(m->d_psf32, n * 4));
	PF_CUDA(ensure(m->d_psfrev32, n * 4));
	PF_CUDA(cudaMemcpy(m->d_psf64.p, m->psf.data(), n * 8, cudaMemcpyHostToDevice));
	PF_CUDA(cudaMemcpy(m->d_psfrev64.p, rev.data(), n * 8, cudaMemcpyHostToDevice));
	PF_CUDA(cudaMemcpy(m->d_psf32.p, f32.data(), n * 4, cudaMemcpyHostToDevice));
	PF_CUDA(cudaMemcpy(m->d_psfrev32.p, r32.data(), n * 4, cudaMemcpyHostToDevice));
	m->psf_dirty = false;
	return PF_OK;
}

// Where the cropped model reads the linear convolution c = psf * src (both
// at the origin of the FFT grid): model(x, y) = c(x + dx, y + dy).
// FFTConvolver returns c at offset_after_convolution (convolve.cpp:270-281):
// src/2, minus one when the source or the kernel is even, less the kernel's
// placement (src - krn)/2 (convolve.cpp:295); the model then crops psf/2
// (model.cpp:307-324).
void fft_offsets(const pf_model *m, const Analysis &a, int &dx, int &dy)
{
	int ox = (int)(a.dw / 2), oy = (int)(a.dh / 2);
	if (a.dw % 2 == 0 || m->psf_w % 2 == 0) ox -= 1;
	if (a.dh % 2 == 0 || m->psf_h % 2 == 0) oy -= 1;
	dx = (int)a.padx + ox - (int)((a.dw - m->psf_w) / 2);
	dy = (int)a.pady + oy - (int)((a.dh - m->psf_h) / 2);
}

// FFT grid and PSF spectra for the "fft" convolver (rebuilt when the PSF or
// the drawing size changes).
int prepare_fft(pf_model *m, const Analysis &a, int batch, bool need32)
{
	const int N = fft_good_size((int)a.dw + (int)m->psf_w - 1);
	const int M = fft_good_size((int)a.dh + (int)m->psf_h - 1);
	if (N > FFT_MAX_LEN || M > FFT_MAX_LEN)
		return set_error(PF_E_INVALID, "image too large for the fft convolver (use brute)");
	const bool resized = m->fft64.M != M || m->fft64.N != N;
	PF_CUDA(m->fft64.setup(M, N));
	const size_t spec = m->fft64.spectrum_elems();
	PF_CUDA(ensure(m->d_kspec64, spec * sizeof(double2)));
	PF_CUDA(ensure(m->d_fftwork64, spec * sizeof(double2) * batch));
	if (resized || m->kspec64_version != m->psf_version) {
		PF_CUDA(m->fft64.set_kernel(m->d_psf64.as<double>(), m->psf_w, m->psf_h, m->d_kspec64.as<double2>(), m->stream));
		m->kspec64_version = m->psf_version;
	}
	if (need32) {
		const bool resized32 = m->fft32.M != M || m->fft32.N != N;
		PF_CUDA(m->fft32.setup(M, N));
		PF_CUDA(ensure(m->d_kspec32, spec * sizeof(float2)));
		PF_CUDA(ensure(m->d_fftwork32, spec * sizeof(float2) * batch));
		if (resized32 || m->kspec32_version != m->psf_version) {
			PF_CUDA(m->fft32.set_kernel(m->d_psf32.as<float>(), m->psf_w, m->psf_h, m->d_kspec32.as<float2>(),
			                            m->stream));
			m->kspec32_version = m->psf_version;
		}
	}
	return PF_OK;
}

// Queue segments per level; capacities start from a pixel-count estimate and
// grow after an overflow.
// kind_groups: the level items are taken kind by kind (models with profiles
// of every kind, launch_levels32), which needs an index buffer beside them.
int prepare_queue(pf_model *m, const Analysis &a, size_t npix_total, QueueSet &q, int32_t *decisions,
                  unsigned long long *level_counts, bool with_masks = false, bool reset = true,
                  bool kind_groups = false)
{
	if (m->caps.size() != (size_t)MAX_LEVELS) {
		m->caps.assign(MAX_LEVELS, 0);
	}
	uint32_t base0 = (uint32_t)std::min<size_t>(std::max<size_t>(npix_total / 4, 4096), 1u << 24);
	for (int l = 0; l < MAX_LEVELS; l++) {
		uint32_t want = l == 0 ? base0 : (l < 3 ? base0 / 2 : 4096);
		if (m->caps[l] < want) m->caps[l] = want;
	}
	size_t total = 0;
	for (int l = 0; l < a.levels; l++) {
		q.off[l] = (uint32_t)total;
		q.cap[l] = m->caps[l];
		total += m->caps[l];
	}
	for (int l = a.levels; l < MAX_LEVELS; l++) {
		q.off[l] = 0;
		q.cap[l] = 0;
	}
	if (total >= (1ull << 32)) return set_error(PF_E_CAPACITY, "subsampling work queue exceeds 2^32 items");
	PF_CUDA(ensure(m->d_items, total * sizeof(SubItem)));
	PF_CUDA(ensure(m->d_ctrl, CTRL_WORDS * 4));
	q.masks = nullptr;
	if (with_masks) {
		PF_CUDA(ensure(m->d_masks, total * MASK_WORDS * sizeof(uint32_t)));
		q.masks = m->d_masks.as<uint32_t>();
	}
	q.perm = nullptr;
	if (kind_groups) {
		PF_CUDA(ensure(m->d_perm, total * sizeof(uint32_t)));
		q.perm = m->d_perm.as<uint32_t>();
	}
	q.items = m->d_items.as<SubItem>();
	q.counts = m->d_ctrl.as<uint32_t>();
	q.overflow = m->d_ctrl.as<uint32_t>() + MAX_LEVELS;
	q.maxres = m->d_ctrl.as<uint32_t>() + MAX_LEVELS + 1;
	q.levels = (uint32_t)a.levels;
	q.decisions = decisions;
	q.level_counts = level_counts;
	// the debug counter buffer holds the evaluation counts after the level counts
	q.evals = level_counts ? level_counts + (size_t)MAX_LEVELS * a.n_profiles : nullptr;
	if (reset) PF_CUDA(cudaMemsetAsync(m->d_ctrl.p, 0, CTRL_WORDS * 4, m->stream));
	return PF_OK;
}

// Reads counts back (after the stream is synchronised) and grows the
// capacities of overflowing levels.  Returns 1 if a retry is needed.
int check_overflow(pf_model *m, const Analysis &a, const uint32_t *ctrl, int &retry)
{
	retry = 0;
	for (int l = 0; l < a.levels; l++) {
		if (ctrl[l] > m->caps[l]) {
			uint64_t want = (uint64_t)ctrl[l] + ctrl[l] / 2 + 1024;
			if (want > (1ull << 30)) return set_error(PF_E_CAPACITY, "subsampling work queue overflow");
			m->caps[l] = (uint32_t)want;
			retry = 1;
		}
	}
	if (ctrl[MAX_LEVELS] & 2u) return set_error(PF_E_CAPACITY, "recursion deeper than the configured levels");
	return PF_OK;
}

int ensure_stream(pf_model *m)
{
	PF_CUDA(cudaSetDevice(m->device));
	return PF_OK;
}

// Upload the derived profile scalars of one parameter set into slot `slot`
// of the device profile array (FP64 form, plus FP32 form when asked).
int derive_and_upload(pf_model *m, const Analysis &a, const std::vector<ProfileParams> &params, int slot,
                      int n_slots, bool fp32)
{
	ModelGeom g = geometry(m, a);
	size_t n = params.size();
	PF_CUDA(ensure(m->h_prof, n * n_slots * sizeof(DevProfile)));
	PF_CUDA(ensure(m->d_prof, n * n_slots * sizeof(DevProfile)));
	DevProfile *hp = m->h_prof.as<DevProfile>() + n * slot;
	if (m->nq.size() < n) m->nq.resize(n);
	for (size_t i = 0; i < n; i++) derive_profile(params[i], g, hp[i], nullptr, shape_memo(m->nq[i], params[i]));
	PF_CUDA(cudaMemcpyAsync(m->d_prof.as<DevProfile>() + n * slot, hp, n * sizeof(DevProfile), cudaMemcpyHostToDevice,
	                        m->stream));
	if (fp32) {
		PF_CUDA(ensure(m->h_fprof, n * n_slots * sizeof(FProfile)));
		PF_CUDA(ensure(m->d_fprof, n * n_slots * sizeof(FProfile)));
		FProfile *hf = m->h_fprof.as<FProfile>() + n * slot;
		for (size_t i = 0; i < n; i++) hf[i] = to_fprofile(hp[i], params[i]);
		PF_CUDA(cudaMemcpyAsync(m->d_fprof.as<FProfile>() + n * slot, hf, n * sizeof(FProfile),
		                        cudaMemcpyHostToDevice, m->stream));
	}
	return PF_OK;
}

// FP32 path, forward: the FP32 drawing images of `batch` proposals to the
// cropped FP64 model images.  The model image is kept in FP64 because the
// residual (data - model) of bright pixels is a small difference of large
// numbers: brute force sums kernel columns in FP64, the "fft" convolver
// transforms in FP64.
// What the FP32 pipeline does beyond one plain crop of the convolved image,
// as run_plain64 does in FP64 (model.cpp:307-334): the drawing-size
// calculation mask for the profiles (draw), the masked convolution's select
// of the unconvolved pixel (sel), the finesampling sum-down (output smaller
// than the crop window) and the output mask (out).  The device masks are
// those upload_masks built for this analysis.
struct Finish32 {
	const uint8_t *draw = nullptr, *sel = nullptr, *out = nullptr;
	bool any = false;
};

Finish32 finish32_of(pf_model *m, const Analysis &a)
{
	Finish32 f;
	if (a.mask) {
		f.draw = m->d_mask_draw.as<uint8_t>();
		if (a.conv && m->conv_kind != CONV_NULL && (a.mask_conv || !m->adjust_mask)) f.sel = f.draw;
		if (a.mask_adjusted && a.ow == m->mask_w && a.oh == m->mask_h) f.out = m->d_mask_out.as<uint8_t>();
	}
	f.any = f.sel || f.out || a.ow != a.cw || a.oh != a.ch;
	return f;
}

// Output (i, j) of the crop window is drawing pixel (i + padx, j + pady); its
// convolution window starts psf/2 before that (0 with the usual padding,
// -psf/2 when a mask let the padding go).
inline int conv_ox(const pf_model *m, const Analysis &a) { return (int)a.padx - (int)(m->psf_w / 2); }
inline int conv_oy(const pf_model *m, const Analysis &a) { return (int)a.pady - (int)(m->psf_h / 2); }

int convolve_crop32(pf_model *m, const Analysis &a, const float *conv, const float *plain, double *model64, int batch,
                    bool conv_on);

int forward_conv32(pf_model *m, const Analysis &a, const float *conv, const float *plain, double *model64, int batch)
{
	const size_t nout = (size_t)a.cw * a.ch;
	const bool conv_on = a.conv && m->conv_kind != CONV_NULL;
	const Finish32 fin = finish32_of(m, a);
	double *dst = model64;  // the crop window, then finished into model64 when needed
	if (fin.any) {
		PF_CUDA(ensure(m->d_model_fine, nout * 8 * batch));
		dst = m->d_model_fine.as<double>();
	}
	PF_TRY(convolve_crop32(m, a, conv, plain, dst, batch, conv_on));
	if (fin.any)
		PF_CUDA(launch_model_finish32(dst, a.cw, a.ch, plain, fin.sel, a.dw, a.dh, a.padx, a.pady, m->fs, fin.out,
		                              model64, a.ow, a.oh, batch, m->stream));
	return PF_OK;
}

// The convolved image plus the unconvolved one on the crop window, FP64.
int convolve_crop32(pf_model *m, const Analysis &a, const float *conv, const float *plain, double *model64, int batch,
                    bool conv_on)
{
	const size_t npix = (size_t)a.dw * a.dh, nout = (size_t)a.cw * a.ch;
	const int ox = conv_ox(m, a), oy = conv_oy(m, a);
	if (conv_on && m->conv_kind == CONV_FFT) {
		PF_TRY(prepare_fft(m, a, batch, false));
		int dx, dy;
		fft_offsets(m, a, dx, dy);
		PF_CUDA(m->fft64.convolve<float, double, float>(conv, a.dw, a.dh, 0, 0, m->d_kspec64.as<double2>(), false,
		                                                m->d_fftwork64.as<double2>(), dx, dy, model64, a.cw, a.ch,
		                                                plain, a.dw, a.padx, a.pady, batch, npix, nout, npix,
		                                                m->stream));
		note_launches(3);
		return PF_OK;
	}
	if (m->precision == PF_FP32_CONV64 || !conv_on) {
		PF_CUDA(ensure(m->d_conv64, npix * 8 * batch));
		PF_CUDA(ensure(m->d_plain64, npix * 8 * batch));
		PF_CUDA(launch_widen(conv, m->d_conv64.as<double>(), npix * batch, m->stream));
		PF_CUDA(launch_widen(plain, m->d_plain64.as<double>(), npix * batch, m->stream));
		for (int b = 0; b < batch; b++) {
			const double *c64 = m->d_conv64.as<double>() + b * npix, *p64 = m->d_plain64.as<double>() + b * npix;
			if (conv_on)
				PF_CUDA(launch_conv64(c64, a.dw, a.dh, ox, oy, m->d_psfrev64.as<double>(), m->psf_w, m->psf_h,
				                      model64 + b * nout, a.cw, a.ch, p64, a.dw, a.padx, a.pady, m->stream));
			else
				PF_CUDA(launch_crop64(c64, a.dw, a.padx, a.pady, model64 + b * nout, a.cw, a.ch, p64, m->stream));
		}
		return PF_OK;
	}
	size_t sb = conv32_scratch_bytes(a.cw, a.ch, batch);
	if (sb) PF_CUDA(ensure(m->d_convsplit, sb));
	PF_CUDA(launch_conv32_to64(conv, a.dw, a.dh, ox, oy, m->d_psfrev32.as<float>(), m->psf_w, m->psf_h, model64,
	                           a.cw, a.ch, plain, a.dw, a.padx, a.pady, batch, (int)npix, (int)nout,
	                           sb ? m->d_convsplit.as<double>() : nullptr, sb, 0, m->stream));
	return PF_OK;
}

// FP32 path, adjoint of the convolution: dlogL/dmodel on the output grid to
// dlogL/d(drawing pixel) of the convolved image, for `batch` proposals.
int adjoint_conv32(pf_model *m, const Analysis &a, const float *wseed, float *gconv, int batch)
{
	const size_t npix = (size_t)a.dw * a.dh, nout = (size_t)a.ow * a.oh;
	if (m->conv_kind == CONV_FFT) {
		PF_TRY(prepare_fft(m, a, batch, false));
		int dx, dy;
		fft_offsets(m, a, dx, dy);
		// g(U) = sum_x w(x) psf(x + d - U): correlation of w placed at d.  The
		// transforms are FP64: FFT roundoff is spread over the whole grid, and
		// in FP32 the error from a bright source's seed swamps the seed of a
		// faint one elsewhere in the field.
		PF_CUDA(m->fft64.convolve<float, float, float>(wseed, a.ow, a.oh, dx, dy, m->d_kspec64.as<double2>(), true,
		                                               m->d_fftwork64.as<double2>(), 0, 0, gconv, a.dw, a.dh, nullptr,
		                                               0, 0, 0, batch, nout, npix, 0, m->stream));
		note_launches(3);
		return PF_OK;
	}
	size_t sb = conv32_scratch_bytes(a.dw, a.dh, batch);
	if (sb) PF_CUDA(ensure(m->d_convsplit, sb));
	// the adjoint of a correlation at offset ox is the correlation with the
	// unreversed PSF at offset 1 - psf - ox
	PF_CUDA(launch_conv32(wseed, a.ow, a.oh, 1 - (int)m->psf_w - conv_ox(m, a), 1 - (int)m->psf_h - conv_oy(m, a),
	                      m->d_psf32.as<float>(), m->psf_w, m->psf_h, gconv, a.dw, a.dh, nullptr, 0, 0, 0, batch,
	                      (int)nout, (int)npix, sb ? m->d_convsplit.as<double>() : nullptr, sb, 0, m->stream));
	return PF_OK;
}

// The adjoint's seeds from dlogL/dmodel (wseed, output grid): g_plain for
// the unconvolved profiles (drawing size) and g_conv for the convolved ones
// (g_conv = g_plain when nothing is convolved).
int adjoint_seed32(pf_model *m, const Analysis &a, const float *wseed, float *&gconv, float *gplain, int batch)
{
	const Finish32 fin = finish32_of(m, a);
	const bool conv_on = a.conv && m->conv_kind != CONV_NULL;
	if (!fin.any) {
		// the seed of the unconvolved image is read by profiles drawn without
		// convolution only (and by every profile when nothing is convolved)
		bool plain = !conv_on;
		for (const auto &p : m->profiles) plain = plain || !p.convolve;
		if (plain)
			PF_CUDA(launch_embed_seed(wseed, a.ow, a.oh, a.padx, a.pady, a.dw, a.dh, batch, gplain, m->stream));
		if (conv_on) PF_TRY(adjoint_conv32(m, a, wseed, gconv, batch));
		else gconv = gplain;
		return PF_OK;
	}
	PF_CUDA(ensure(m->d_seed_fine, (size_t)a.cw * a.ch * 4 * batch));
	float *seed = m->d_seed_fine.as<float>();
	PF_CUDA(launch_seed_finish32(wseed, a.ow, a.oh, fin.out, fin.sel, m->fs, a.cw, a.ch, a.padx, a.pady, a.dw, a.dh,
	                             batch, seed, gplain, m->stream));
	if (conv_on) {
		Analysis af = a;  // the seed of the convolution lives on the fine crop window
		af.ow = a.cw;
		af.oh = a.ch;
		PF_TRY(adjoint_conv32(m, af, seed, gconv, batch));
	}
	else {
		gconv = gplain;
	}
	return PF_OK;
}

// FP64 model image into d_model64 (out dims), queue-overflow checked by caller.
int run_plain64(pf_model *m, const Analysis &a, const DevProfile *dprof, QueueSet &q)
{
	size_t npix = (size_t)a.dw * a.dh;
	PF_CUDA(ensure(m->d_conv64, npix * 8));
	PF_CUDA(ensure(m->d_plain64, npix * 8));
	PF_CUDA(ensure(m->d_model64, (size_t)a.cw * a.ch * 8 + 8));
	double *conv = m->d_conv64.as<double>(), *plain = m->d_plain64.as<double>();
	PF_TRY(upload_masks(m, a));
	const uint8_t *mask = a.mask ? m->d_mask_draw.as<uint8_t>() : nullptr;
	PF_CUDA(launch_pixels64(dprof, a.n_profiles, a.dw, a.dh, m->sx / m->fs, m->sy / m->fs, conv, plain, mask, q,
	                        m->stream));
	for (int p = 0; p < a.n_profiles; p++) {
		if (m->profiles[p].kind == PK_PSF) {
			PF_CUDA(launch_psf_stamp64(dprof, p, m->d_psf64.as<double>(), m->psf_w, m->psf_h, m->psf_sx, m->psf_sy,
			                           m->sx / m->fs, m->sy / m->fs, a.padx, a.pady, a.dw, a.dh, conv, plain,
			                           m->stream));
		}
	}
	PF_CUDA(launch_levels64(dprof, a.levels, conv, plain, q, m->stream));
	if (q.decisions) PF_CUDA(launch_count_decisions(q, a.levels, npix, m->stream));
	PF_CUDA(record_event(m->ev[1], m->stream));

	double *model = m->d_model64.as<double>();
	if (a.conv && m->conv_kind == CONV_FFT) {
		PF_TRY(prepare_fft(m, a, 1, false));
		int dx, dy;
		fft_offsets(m, a, dx, dy);
		PF_CUDA(m->fft64.convolve<double, double, double>(conv, a.dw, a.dh, 0, 0, m->d_kspec64.as<double2>(), false,
		                                                  m->d_fftwork64.as<double2>(), dx, dy, model, a.cw, a.ch,
		                                                  plain, a.dw, a.padx, a.pady, 1, 0, 0, 0, m->stream));
		note_launches(3);
	}
	else if (a.conv && m->conv_kind != CONV_NULL) {
		// output (i, j) is drawing pixel (i + padx, j + pady); its window starts
		// psf/2 before that (0 with the usual padding, -psf/2 when a mask let the
		// padding go)
		const int ox = (int)a.padx - (int)(m->psf_w / 2), oy = (int)a.pady - (int)(m->psf_h / 2);
		PF_CUDA(launch_conv64(conv, a.dw, a.dh, ox, oy, m->d_psfrev64.as<double>(), m->psf_w, m->psf_h, model, a.cw,
		                      a.ch, plain, a.dw, a.padx, a.pady, m->stream));
	}
	else {
		PF_CUDA(launch_crop64(conv, a.dw, a.padx, a.pady, model, a.cw, a.ch, plain, m->stream));
	}
	if (a.conv && a.mask && m->conv_kind != CONV_NULL && (a.mask_conv || !m->adjust_mask))
		PF_CUDA(launch_mask_select64(model, a.cw, a.ch, plain, m->d_mask_draw.as<uint8_t>(), a.dw, a.padx, a.pady,
		                             m->stream));
	if (a.ow != a.cw || a.oh != a.ch) {
		// finesampled output summed down (model.cpp:326-329); reuse conv as scratch
		PF_CUDA(cudaMemcpyAsync(conv, model, (size_t)a.cw * a.ch * 8, cudaMemcpyDeviceToDevice, m->stream));
		PF_CUDA(launch_downsample64(conv, a.cw, a.ch, m->fs, model, a.ow, a.oh, m->stream));
	}
	// image &= mask when the mask was adjusted (model.cpp:330-334); the user's
	// mask has the output's size unless the finesampled image is returned
	if (a.mask_adjusted && a.ow == m->mask_w && a.oh == m->mask_h)
		PF_CUDA(launch_mask_and64(model, m->d_mask_out.as<uint8_t>(), (size_t)a.ow * a.oh, m->stream));
	PF_CUDA(record_event(m->ev[2], m->stream));
	return PF_OK;
}

int fetch_debug(pf_model *m, const Analysis &a)
{
	size_t npix = (size_t)a.dw * a.dh;
	m->decisions.resize(npix * a.n_profiles);
	m->level_counts.resize((size_t)MAX_LEVELS * a.n_profiles);
	m->evals.resize((size_t)(1 + MAX_LEVELS) * a.n_profiles);
	PF_CUDA(cudaMemcpyAsync(m->decisions.data(), m->d_decisions.p, npix * a.n_profiles * 4, cudaMemcpyDeviceToHost,
	                        m->stream));
	PF_CUDA(cudaMemcpyAsync(m->level_counts.data(), m->d_level_counts.p, (size_t)MAX_LEVELS * a.n_profiles * 8,
	                        cudaMemcpyDeviceToHost, m->stream));
	PF_CUDA(cudaMemcpyAsync(m->evals.data(), m->d_level_counts.as<unsigned long long>() + (size_t)MAX_LEVELS * a.n_profiles,
	                        (size_t)(1 + MAX_LEVELS) * a.n_profiles * 8, cudaMemcpyDeviceToHost, m->stream));
	PF_CUDA(cudaStreamSynchronize(m->stream));
	m->dec_npix = (unsigned)npix;
	m->dec_levels = a.levels;
	return PF_OK;
}

// Full FP64 evaluation into d_model64 with retries on queue overflow.
int evaluate64(pf_model *m, Analysis &a)
{
	PF_TRY(ensure_stream(m));
	PF_TRY(analyze(m, a));
	PF_TRY(upload_psf(m));
	PF_CUDA(record_event(m->ev[0], m->stream));
	PF_TRY(derive_and_upload(m, a, m->profiles, 0, 1, false));
	size_t npix = (size_t)a.dw * a.dh;
	PF_CUDA(ensure(m->h_ctrl, CTRL_WORDS * 4));
	for (int attempt = 0; attempt < 8; attempt++) {
		int32_t *dec = nullptr;
		unsigned long long *lc = nullptr;
		if (m->debug) {
			PF_CUDA(ensure(m->d_decisions, npix * a.n_profiles * 4));
			const size_t counter_bytes = (size_t)(2 * MAX_LEVELS + 1) * a.n_profiles * 8;  // level counts, evaluations
			PF_CUDA(ensure(m->d_level_counts, counter_bytes));
			PF_CUDA(cudaMemsetAsync(m->d_decisions.p, 0, npix * a.n_profiles * 4, m->stream));
			PF_CUDA(cudaMemsetAsync(m->d_level_counts.p, 0, counter_bytes, m->stream));
			dec = m->d_decisions.as<int32_t>();
			lc = m->d_level_counts.as<unsigned long long>();
		}
		QueueSet q;
		PF_TRY(prepare_queue(m, a, npix * a.n_profiles, q, dec, lc));
		PF_TRY(run_plain64(m, a, m->d_prof.as<DevProfile>(), q));
		PF_CUDA(cudaMemcpyAsync(m->h_ctrl.p, m->d_ctrl.p, CTRL_WORDS * 4, cudaMemcpyDeviceToHost, m->stream));
		PF_CUDA(cudaStreamSynchronize(m->stream));
		int retry = 0;
		PF_TRY(check_overflow(m, a, m->h_ctrl.as<uint32_t>(), retry));
		if (!retry) {
			if (m->debug) PF_TRY(fetch_debug(m, a));
			float t = 0;
			cudaEventElapsedTime(&t, m->ev[0], m->ev[2]);
			m->timings_lazy = false;
			m->timings[0] = t;
			cudaEventElapsedTime(&m->timings[1], m->ev[0], m->ev[1]);
			cudaEventElapsedTime(&m->timings[2], m->ev[1], m->ev[2]);
			cudaGetLastError();
			return PF_OK;
		}
	}
	return set_error(PF_E_CAPACITY, "subsampling work queue kept overflowing");
}

// ---------------------------------------------------------------------------
// FP32 path with forward tangents and the adjoint reduction
// ---------------------------------------------------------------------------

// The model's likelihood (pf_model_set_likelihood) of `batch` images against
// its data, with the adjoint seed when wseed is given.
// Ticket words of the one-launch norm likelihood, one per image: zeroed when
// the buffer is (re)allocated, left at zero by every launch.
int like_tickets(pf_model *m, int batch, unsigned **tickets)
{
	void *before = m->d_like_tickets.p;
	PF_CUDA(ensure(m->d_like_tickets, (size_t)batch * sizeof(unsigned)));
	if (m->d_like_tickets.p != before)
		PF_CUDA(cudaMemsetAsync(m->d_like_tickets.p, 0, m->d_like_tickets.bytes, m->stream));
	*tickets = m->d_like_tickets.as<unsigned>();
	return PF_OK;
}

int enqueue_like(pf_model *m, const double *model64, int nout, int batch, double *out, float *wseed, cudaStream_t s)
{
	PF_CUDA(ensure(m->d_partials, (size_t)NPARTS * batch * 2 * sizeof(double2)));
	PF_CUDA(ensure(m->d_likestats, (size_t)batch * LIKE_SCRATCH_PER_IMAGE * 8));
	unsigned *tickets = nullptr;
	if (m->like_kind == LIKE_NORM) PF_TRY(like_tickets(m, batch, &tickets));
	PF_CUDA(launch_like64(m->like_kind, model64, m->d_data.as<double>(), m->d_sigma.as<double>(),
	                      m->has_region ? m->d_region.as<uint8_t>() : nullptr, nout, batch, 0,
	                      m->d_partials.as<double2>(), like_parts(nout, batch), m->d_likestats.as<double>(), out,
	                      wseed, s, tickets));
	return PF_OK;
}

// Tangent planes kept per radial profile: the most any profile of the model
// fills (9 for Sersic and Moffat models, up to 12 with core-Sersic).
int tangent_stride(const pf_model *m)
{
	int nt = NTAN_GEOM + 3;
	for (auto &p : m->profiles)
		if (is_radial_kind(p.kind)) nt = std::max(nt, tangent_count(p.kind));
	return nt;
}

bool has_psf_profile(const pf_model *m)
{
	for (auto &p : m->profiles)
		if (p.kind == PK_PSF) return true;
	return false;
}

// Sersic profiles with adjust: those whose centre cusp may recurse past
// level 2 (the count picks how the deep levels are launched).
int cusp_count(const pf_model *m)
{
	int n = 0;
	for (auto &p : m->profiles)
		if (p.kind == PK_SERSIC && p.adjust) n++;
	return n;
}

// Whether the model has radial profiles beyond Sersic and Moffat (selects the
// FP32 kernels that carry every kind's tangents).
bool all_kinds(const pf_model *m)
{
	for (auto &p : m->profiles)
		if (is_radial_kind(p.kind) && p.kind != PK_SERSIC && p.kind != PK_MOFFAT) return true;
	return false;
}

// Scratch of launch_jac_reduce for n_profiles profiles on a width x height drawing; the
// tickets (one per profile and one for the folded gradient step) start at
// zero when allocated and the kernel leaves them at zero.
int jac_scratch(pf_model *m, unsigned width, unsigned height, int n_profiles, double **partials, unsigned **tickets)
{
	const size_t pb = (size_t)n_profiles * jac_reduce_blocks(width, height, n_profiles) * NTAN * sizeof(double);
	PF_CUDA(ensure(m->d_jac_partials, pb));
	void *before = m->d_jac_tickets.p;
	PF_CUDA(ensure(m->d_jac_tickets, (size_t)(n_profiles + 1) * sizeof(unsigned)));
	if (m->d_jac_tickets.p != before) PF_CUDA(cudaMemsetAsync(m->d_jac_tickets.p, 0, m->d_jac_tickets.bytes, m->stream));
	*partials = m->d_jac_partials.as<double>();
	*tickets = m->d_jac_tickets.as<unsigned>();
	return PF_OK;
}

// Events of the FP32 pipeline.  Outside a capture each is recorded on the
// stream.  A captured graph keeps only the inner phase events ev[1] and
// ev[2], and only with phase timing on: the caller records ev[0] and ev[3]
// on the stream around the graph's launch.
cudaError_t phase_event(pf_model *m, int i, cudaStream_t s)
{
	cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
	cudaStreamIsCapturing(s, &st);
	if (st != cudaStreamCaptureStatusActive) return cudaEventRecord(m->ev[i], s);
	if ((i == 1 || i == 2) && m->phase_timing) return cudaEventRecordWithFlags(m->ev[i], s, cudaEventRecordExternal);
	return cudaSuccess;
}

// Launches a recorded FP32 pipeline between the outer timing events.
cudaError_t launch_recorded(pf_model *m, cudaGraphExec_t g)
{
	cudaError_t e = cudaEventRecord(m->ev[0], m->stream);
	if (e == cudaSuccess) e = cudaGraphLaunch(g, m->stream);
	if (e == cudaSuccess) e = cudaEventRecord(m->ev[3], m->stream);
	m->phases_recorded = m->phase_timing;
	return e;
}

int run_fp32(pf_model *m, const Analysis &a, const FProfile *fprof, QueueSet &q, bool want_grad, double *d_out)
{
	size_t npix = (size_t)a.dw * a.dh;
	size_t nout = (size_t)a.ow * a.oh;
	int nprof = a.n_profiles;
	PF_CUDA(ensure(m->d_conv32, npix * 4));
	PF_CUDA(ensure(m->d_plain32, npix * 4));
	PF_CUDA(ensure(m->d_model32, (size_t)a.cw * a.ch * 4 + 4));
	float *jac = nullptr;
	if (want_grad) {
		PF_CUDA(ensure(m->d_jac, npix * tangent_stride(m) * nprof * 4));
		jac = m->d_jac.as<float>();
	}
	float *conv = m->d_conv32.as<float>(), *plain = m->d_plain32.as<float>(), *model = m->d_model32.as<float>();
	PF_CUDA(launch_pixels32(fprof, m->d_prof_begin.as<int>(), 1, a.dw, a.dh, m->sx / m->fs, m->sy / m->fs, conv, plain,
	                        jac, tangent_stride(m), all_kinds(m), q, m->stream, finish32_of(m, a).draw));
	PF_CUDA(launch_levels32(fprof, a.levels, (unsigned)npix, conv, plain, jac, tangent_stride(m), all_kinds(m),
	                        cusp_count(m), q,
	                        m->stream));
	if (has_psf_profile(m))
		PF_CUDA(launch_psf_stamp32(m->d_prof.as<DevProfile>(), m->d_prof_begin.as<int>(), 1, m->d_psf64.as<double>(),
		                           m->psf_w, m->psf_h, m->psf_sx, m->psf_sy, m->sx / m->fs, m->sy / m->fs, a.padx,
		                           a.pady, a.dw, a.dh, conv, plain, m->stream));
	PF_CUDA(phase_event(m, 1, m->stream));
	PF_CUDA(ensure(m->d_model64, (size_t)a.cw * a.ch * 8 + 8));
	double *model64 = m->d_model64.as<double>();
	PF_TRY(forward_conv32(m, a, conv, plain, model64, 1));
	(void)model;
	PF_CUDA(phase_event(m, 2, m->stream));
	if (!m->has_data) return PF_OK;
	float *wseed = nullptr;
	if (want_grad) {
		PF_CUDA(ensure(m->d_wseed, nout * 4));
		wseed = m->d_wseed.as<float>();
	}
	PF_TRY(enqueue_like(m, model64, (int)nout, 1, d_out + ResultLayout::LL, wseed, m->stream));
	if (want_grad) {
		PF_CUDA(ensure(m->d_gconv, npix * 4));
		PF_CUDA(ensure(m->d_gplain, npix * 4));
		float *gconv = m->d_gconv.as<float>(), *gplain = m->d_gplain.as<float>();
		PF_TRY(adjoint_seed32(m, a, wseed, gconv, gplain, 1));
		PF_CUDA(cudaMemsetAsync(d_out + ResultLayout::T0, 0, (size_t)nprof * NTAN * 8, m->stream));
		double *jpart;
		unsigned *jtick;
		PF_TRY(jac_scratch(m, a.dw, a.dh, nprof, &jpart, &jtick));
		PF_CUDA(launch_jac_reduce(jac, gconv, gplain, fprof, m->d_prof_batch.as<int>(), nprof, a.dw, a.dh,
		                          m->sx / m->fs, m->sy / m->fs, tangent_stride(m), jpart, jtick,
		                          d_out + ResultLayout::T0, m->stream));
		if (has_psf_profile(m))
			PF_CUDA(launch_psf_adjoint32(m->d_prof.as<DevProfile>(), m->d_prof_begin.as<int>(), 1, nprof,
			                             m->d_psf64.as<double>(), m->psf_w, m->psf_h, m->psf_sx, m->psf_sy,
			                             m->sx / m->fs, m->sy / m->fs, a.padx, a.pady, a.dw, a.dh, gconv, gplain,
			                             d_out + ResultLayout::T0, m->stream));
	}
	PF_CUDA(phase_event(m, 3, m->stream));
	return PF_OK;
}

// Everything one FP32 evaluation puts on the stream, from the upload of the
// staged profile scalars to the download of logL, tangent reductions and
// queue counters.  Run eagerly, or captured once and replayed as a graph.
int enqueue_fp32(pf_model *m, const Analysis &a, bool want_grad, size_t nres, QueueSet &q)
{
	size_t n = (size_t)a.n_profiles;
	PF_CUDA(phase_event(m, 0, m->stream));
	PF_CUDA(cudaMemcpyAsync(m->d_fprof.p, m->h_fprof.p, n * sizeof(FProfile), cudaMemcpyHostToDevice, m->stream));
	if (has_psf_profile(m))  // the psf stamp reads the FP64 records
		PF_CUDA(cudaMemcpyAsync(m->d_prof.p, m->h_prof.p, n * sizeof(DevProfile), cudaMemcpyHostToDevice, m->stream));
	PF_CUDA(cudaMemsetAsync(m->d_ctrl.p, 0, CTRL_WORDS * 4, m->stream));
	PF_TRY(run_fp32(m, a, m->d_fprof.as<FProfile>(), q, want_grad, m->d_results.as<double>()));
	char *hr = m->h_results.as<char>();
	PF_CUDA(cudaMemcpyAsync(hr, m->d_results.p, nres * 8, cudaMemcpyDeviceToHost, m->stream));
	PF_CUDA(cudaMemcpyAsync(hr + nres * 8, m->d_ctrl.p, CTRL_WORDS * 4, cudaMemcpyDeviceToHost, m->stream));
	return PF_OK;
}

void drop_graph(pf_model *m)
{
	if (m->graph_exec) cudaGraphExecDestroy(m->graph_exec);
	m->graph_exec = nullptr;
	m->graph_sig.clear();
}

// What a captured graph depends on: sizes, queue layout and buffer addresses.
std::vector<uint64_t> graph_signature(pf_model *m, const Analysis &a, bool want_grad, const QueueSet &q)
{
	std::vector<uint64_t> s = {a.dw, a.dh, a.ow, a.oh, (uint64_t)a.n_profiles, (uint64_t)a.levels, a.conv,
	                           (uint64_t)m->conv_kind, (uint64_t)m->precision, m->psf_w, m->psf_h, m->has_data,
	                           m->has_region, want_grad, (uint64_t)m->like_kind, (uint64_t)m->phase_timing};
	for (int l = 0; l < a.levels; l++) s.push_back(((uint64_t)q.off[l] << 32) | q.cap[l]);
	const DevBuf *bufs[] = {&m->d_fprof, &m->d_prof_begin, &m->d_prof_batch, &m->d_conv32, &m->d_plain32,
	                        &m->d_model64, &m->d_conv64, &m->d_plain64, &m->d_jac, &m->d_gconv, &m->d_gplain,
	                        &m->d_wseed, &m->d_items, &m->d_ctrl, &m->d_partials, &m->d_results, &m->d_psf32,
	                        &m->d_psfrev32, &m->d_psfrev64, &m->d_data, &m->d_sigma, &m->d_region, &m->d_convsplit, &m->d_jac_partials, &m->d_jac_tickets, &m->d_likestats, &m->d_like_tickets};
	for (auto *b : bufs) s.push_back((uint64_t)(uintptr_t)b->p);
	// calculation mask and finesampling steps (finish32_of) and their buffers
	for (const DevBuf *b : {&m->d_mask_draw, &m->d_mask_out, &m->d_model_fine, &m->d_seed_fine, &m->d_perm})
		s.push_back((uint64_t)(uintptr_t)b->p);
	s.push_back(((uint64_t)a.mask << 0) | ((uint64_t)a.mask_conv << 1) | ((uint64_t)a.mask_adjusted << 2) |
	            ((uint64_t)m->adjust_mask << 3) | ((uint64_t)m->fs << 8) | ((uint64_t)a.cw << 24));
	s.push_back(((uint64_t)a.ch << 32) | ((uint64_t)m->mask_w << 16) | m->mask_h);
	s.push_back(((uint64_t)a.padx << 32) | a.pady);
	s.push_back((uint64_t)m->profiles.size());
	for (const DevBuf *b : {&m->d_prof, &m->d_psf64}) s.push_back((uint64_t)(uintptr_t)b->p);
	// which kernels run: AK variants and psf stamps by kind, the seed of the
	// unconvolved image when a profile is drawn without convolution
	for (auto &p : m->profiles) s.push_back((uint64_t)p.kind | ((uint64_t)(p.convolve ? 1 : 0) << 32));
	s.push_back((uint64_t)(uintptr_t)m->h_results.p);
	return s;
}

// The FP32 pipeline's phase times are read from its events only when asked
// for (pf_model_last_timings), which keeps the event queries off the
// evaluation's own path.
void finish_timings32(pf_model *m) { m->timings_lazy = true; }

void resolve_timings32(pf_model *m)
{
	m->timings_lazy = false;
	// (a polled call returns before its closing event has been recorded)
	cudaEventSynchronize(m->has_data ? m->ev[3] : m->ev[2]);
	if (m->phases_recorded) {
		cudaEventElapsedTime(&m->timings[1], m->ev[0], m->ev[1]);
		cudaEventElapsedTime(&m->timings[2], m->ev[1], m->ev[2]);
	}
	else {
		m->timings[1] = m->timings[2] = m->timings[3] = NAN;
	}
	if (m->has_data) {
		if (m->phases_recorded) cudaEventElapsedTime(&m->timings[3], m->ev[2], m->ev[3]);
		cudaEventElapsedTime(&m->timings[0], m->ev[0], m->ev[3]);
	}
	else {
		cudaEventElapsedTime(&m->timings[0], m->ev[0], m->ev[2]);
	}
	cudaGetLastError();  // a timing failure must not surface as a later launch error
}

int evaluate32(pf_model *m, Analysis &a, bool want_grad, std::vector<double> *results)
{
	PF_TRY(ensure_stream(m));
	PF_TRY(analyze(m, a));
	if (m->has_data && (m->data_w != a.ow || m->data_h != a.oh))
		return set_error(PF_E_STATE, "data dimensions differ from the model's output dimensions");
	PF_TRY(upload_psf(m));
	PF_TRY(upload_masks(m, a));  // before any capture: it copies synchronously when the mask changed
	int nprof = a.n_profiles;
	// profile scalars, staged in pinned memory (the upload is part of the pipeline)
	{
		ModelGeom g = geometry(m, a);
		PF_CUDA(ensure(m->h_prof, nprof * sizeof(DevProfile)));
		PF_CUDA(ensure(m->d_prof, nprof * sizeof(DevProfile)));
		PF_CUDA(ensure(m->h_fprof, nprof * sizeof(FProfile)));
		PF_CUDA(ensure(m->d_fprof, nprof * sizeof(FProfile)));
		DevProfile *hp = m->h_prof.as<DevProfile>();
		FProfile *hf = m->h_fprof.as<FProfile>();
		if ((int)m->nq.size() < nprof) m->nq.resize(nprof);
		for (int i = 0; i < nprof; i++) {
			derive_profile(m->profiles[i], g, hp[i], nullptr, shape_memo(m->nq[i], m->profiles[i]));
			hf[i] = to_fprofile(hp[i], m->profiles[i]);
		}
	}
	if (m->prof_begin_n != nprof) {
		std::vector<int> begin = {0, nprof};
		std::vector<int> batch(nprof, 0);
		PF_CUDA(ensure(m->d_prof_begin, 2 * 4));
		PF_CUDA(ensure(m->d_prof_batch, nprof * 4));
		PF_CUDA(cudaMemcpy(m->d_prof_begin.p, begin.data(), 8, cudaMemcpyHostToDevice));
		PF_CUDA(cudaMemcpy(m->d_prof_batch.p, batch.data(), nprof * 4, cudaMemcpyHostToDevice));
		m->prof_begin_n = nprof;
	}
	size_t nres = ResultLayout::T0 + (size_t)nprof * NTAN;
	PF_CUDA(ensure(m->d_results, nres * 8));
	PF_CUDA(ensure(m->h_results, nres * 8 + CTRL_WORDS * 4));
	size_t npix = (size_t)a.dw * a.dh;
	char *hr = m->h_results.as<char>();

	for (int attempt = 0; attempt < 8; attempt++) {
		QueueSet q;
		PF_TRY(prepare_queue(m, a, npix * nprof, q, nullptr, nullptr, false, true, all_kinds(m)));
		bool replayed = false;
		if (want_grad && m->graph_exec && m->graph_sig == graph_signature(m, a, want_grad, q)) {
			PF_CUDA(launch_recorded(m, m->graph_exec));
			note_launches((int)m->graph_kernels);
			replayed = true;
		}
		else {
			PF_TRY(enqueue_fp32(m, a, want_grad, nres, q));
			m->phases_recorded = true;
		}
		PF_CUDA(cudaStreamSynchronize(m->stream));
		int retry = 0;
		PF_TRY(check_overflow(m, a, reinterpret_cast<uint32_t *>(hr + nres * 8), retry));
		if (retry) {
			drop_graph(m);
			continue;
		}
		if (results) results->assign(reinterpret_cast<double *>(hr), reinterpret_cast<double *>(hr) + nres);
		finish_timings32(m);
		if (want_grad && !replayed && m->use_graphs) {
			// capture the pipeline that just ran for the next evaluations
			drop_graph(m);
			unsigned long long before = g_launches.load();
			cudaGraph_t graph = nullptr;
			PF_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
			int st = enqueue_fp32(m, a, want_grad, nres, q);
			cudaError_t ce = cudaStreamEndCapture(m->stream, &graph);
			m->graph_kernels = g_launches.load() - before;
			g_launches -= m->graph_kernels;
			if (st == PF_OK && ce == cudaSuccess && graph) {
				if (cudaGraphInstantiate(&m->graph_exec, graph, 0) == cudaSuccess)
					m->graph_sig = graph_signature(m, a, want_grad, q);
				else
					m->graph_exec = nullptr;
			}
			if (graph) cudaGraphDestroy(graph);
			cudaGetLastError();
		}
		return PF_OK;
	}
	return set_error(PF_E_CAPACITY, "subsampling work queue kept overflowing");
}

// d logL / d parameter from the tangent reductions T[0..8] of one profile.
int gradient_code(const ProfileParams &p, const char *name, int &code);
int check_profile(pf_model *m, int index);

// ---------------------------------------------------------------------------
// Batched FP32 likelihood + adjoint gradient: B proposals of the model (its
// profiles with the listed parameters replaced by values[b][.]), all against
// the model's data.  The scalar prologue runs on the device, proposals are
// processed in chunks that fit the memory budget, and each chunk's pipeline
// is replayed from a CUDA graph after its first run.
// ---------------------------------------------------------------------------

}  // namespace

// Host-prologue staging: one pinned block [DevProfile x n | FProfile x n |
// invalid flags x C] uploaded with one copy; results [logL x C | gradient x
// C*nrefs | queue counters] downloaded with one copy.
inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
// Largest staged upload read by launch_stage_in instead of a copy.
constexpr size_t STAGE_IN_MAX_BYTES = 64 << 10;

struct StageLayout {
	size_t f = 0, inv = 0, seq = 0, total = 0;
	StageLayout(int C, int nprof)
	{
		f = align256((size_t)C * nprof * sizeof(DevProfile));
		inv = f + align256((size_t)C * nprof * sizeof(FProfile));
		seq = inv + align256((size_t)C * 4);  // the call's sequence number (completion word)
		total = seq + 256;
	}
};

// The completion word behind the results and queue counters in the pinned
// result buffer.
inline size_t out_flag_offset(int C, int nrefs) { return align256((size_t)C * (1 + nrefs) * 8 + CTRL_WORDS * 4); }

// A batch evaluated in ProFit's fit space (pf_model_lp_grad_batch): the
// proposals are fitted vectors parm (nfit per row) instead of model values.
struct FitRun {
	FitSpaceView host;  // entries in host memory (few-proposal path)
	FitSpaceView dev;   // entries in device memory
	double *lp, *grad, *parm_out, *ll;  // caller's outputs (any but lp may be null)
};

struct BatchState {
	DevBuf d_tmpl, d_refs, d_values, d_dev, d_invalid, d_out, d_ll, d_T, d_stage;
	HostBuf h_tmpl, h_values, h_out, h_stage;
	// fit space: parm of the chunk, [C] LP, [C][nfit] gradient, [C] LL, [C][nfit] parm_out
	DevBuf d_fit_parm, d_fit_out;
	HostBuf h_fit_out;
	void *h_stage_dev = nullptr;  // h_stage as the device addresses it (mapped pinned memory), or null
	void *h_out_dev = nullptr;    // likewise h_out
	int refs_n = -1, chunk = 0;
	std::vector<int> refs_host;
	// (profile, kind, rescale_flux, name) of the references refs_host was resolved for
	std::vector<std::tuple<int, int, int, std::string>> refs_key;
	cudaGraphExec_t graph = nullptr;
	std::vector<uint64_t> sig;
	unsigned long long graph_kernels = 0;
	// the pipeline ends by storing the call's sequence number into the
	// result buffer (set by enqueue_batch_chunk); seq counts the calls
	bool polled = false;
	unsigned seq = 0;
	~BatchState()
	{
		if (graph) cudaGraphExecDestroy(graph);
	}
};

namespace {

constexpr size_t BATCH_BUDGET_BYTES = 24ull << 30;

// A few proposals: the scalar prologue (qgamma's Newton iterations are one
// long dependent FP64 chain) is faster on the host than in one GPU thread.
// Many proposals: one GPU thread per (proposal, profile) runs them in parallel.
constexpr int HOST_PROLOGUE_MAX = 16;

int enqueue_batch_chunk(pf_model *m, BatchState &bs, const Analysis &a, int C, int nrefs, const QueueSet &q,
                        bool host_prologue, bool recompute, const FitRun *fit)
{
	const int nprof = a.n_profiles;
	const size_t npix = (size_t)a.dw * a.dh, nout = (size_t)a.ow * a.oh;
	cudaStream_t s = m->stream;
	float *conv = m->d_conv32.as<float>(), *plain = m->d_plain32.as<float>();
	float *jac = recompute ? nullptr : m->d_jac.as<float>();
	double *model64 = m->d_model64.as<double>();
	float *wseed = m->d_wseed.as<float>(), *gconv = m->d_gconv.as<float>(), *gplain = m->d_gplain.as<float>();
	const int *ref_profile = bs.d_refs.as<int>(), *ref_offset = ref_profile + nrefs, *ref_code = ref_offset + nrefs;

	const StageLayout L(C, nprof);
	const DevProfile *dev = host_prologue ? bs.d_stage.as<DevProfile>() : bs.d_dev.as<DevProfile>();
	const FProfile *fprof = host_prologue ? reinterpret_cast<const FProfile *>(bs.d_stage.as<char>() + L.f)
	                                      : m->d_fprof.as<FProfile>();
	const int *invalid = host_prologue ? reinterpret_cast<const int *>(bs.d_stage.as<char>() + L.inv)
	                                   : bs.d_invalid.as<int>();
	double *out_ll = bs.d_out.as<double>(), *out_grad = out_ll + C;

	PF_CUDA(phase_event(m, 0, s));
	// a small stage is read by a kernel straight from the pinned buffer, which
	// also zeroes the queue counters (one programmatic launch instead of a
	// memset and a copy); a large one goes by copy
	void *hmap = host_prologue && L.total <= STAGE_IN_MAX_BYTES ? bs.h_stage_dev : nullptr;
	if (hmap) {
		PF_CUDA(launch_stage_in(bs.d_stage.p, hmap, L.total, q.counts, CTRL_WORDS, s));
	}
	else {
		PF_CUDA(cudaMemsetAsync(q.counts, 0, CTRL_WORDS * 4, s));
		if (host_prologue) PF_CUDA(cudaMemcpyAsync(bs.d_stage.p, bs.h_stage.p, L.total, cudaMemcpyHostToDevice, s));
	}
	// the recomputing adjoint accumulates the tangent sums with atomics; the
	// stored-plane reduction writes every slot the gradient reads
	if (recompute) PF_CUDA(cudaMemsetAsync(bs.d_T.p, 0, (size_t)C * nprof * NTAN * 8, s));
	if (!host_prologue) {
		PF_CUDA(cudaMemcpyAsync(bs.d_tmpl.p, bs.h_tmpl.p, nprof * sizeof(ProfileParams), cudaMemcpyHostToDevice, s));
		if (fit) {
			// the fitted vectors in, the model values of the proposals from them
			const int nfit = fit->dev.nfit;
			PF_CUDA(cudaMemcpyAsync(bs.d_fit_parm.p, bs.h_values.p, (size_t)C * nfit * 8, cudaMemcpyHostToDevice, s));
			PF_CUDA(launch_fit_remake(fit->dev, C, bs.d_fit_parm.as<double>(), bs.d_values.as<double>(),
			                          bs.d_fit_out.as<double>() + (size_t)C * (2 + nfit), s));
		}
		else {
			PF_CUDA(cudaMemcpyAsync(bs.d_values.p, bs.h_values.p, (size_t)C * nrefs * 8, cudaMemcpyHostToDevice, s));
		}
		PF_CUDA(cudaMemsetAsync(bs.d_invalid.p, 0, (size_t)C * 4, s));
		PF_CUDA(launch_batch_prologue(bs.d_tmpl.as<ProfileParams>(), nprof, C, ref_profile, ref_offset, nrefs,
		                              bs.d_values.as<double>(), geometry(m, a), bs.d_dev.as<DevProfile>(),
		                              m->d_fprof.as<FProfile>(), bs.d_invalid.as<int>(), s));
	}
	const int nt = tangent_stride(m);
	const bool ak = all_kinds(m);
	const Finish32 fin = finish32_of(m, a);
	PF_CUDA(launch_pixels32(fprof, m->d_prof_begin.as<int>(), C, a.dw, a.dh, m->sx / m->fs, m->sy / m->fs, conv, plain,
	                        jac, nt, ak, q, s, fin.draw));
	PF_CUDA(launch_levels32(fprof, a.levels, (unsigned)npix, conv, plain, jac, nt, ak, C * cusp_count(m), q, s));
	if (has_psf_profile(m))
		PF_CUDA(launch_psf_stamp32(dev, m->d_prof_begin.as<int>(), C, m->d_psf64.as<double>(), m->psf_w, m->psf_h,
		                           m->psf_sx, m->psf_sy, m->sx / m->fs, m->sy / m->fs, a.padx, a.pady, a.dw, a.dh,
		                           conv, plain, s));
	PF_CUDA(phase_event(m, 1, s));
	PF_TRY(forward_conv32(m, a, conv, plain, model64, C));
	PF_CUDA(phase_event(m, 2, s));
	PF_TRY(enqueue_like(m, model64, (int)nout, C, bs.d_ll.as<double>(), wseed, s));
	PF_TRY(adjoint_seed32(m, a, wseed, gconv, gplain, C));
	if (recompute)
		PF_CUDA(launch_adjoint_recompute(fprof, m->d_prof_batch.as<int>(), m->d_prof_begin.as<int>(), C, C * nprof,
		                                 a.dw, a.dh, m->sx / m->fs,
		                                 m->sy / m->fs, gconv, gplain, a.levels, ak, q, bs.d_T.as<double>(), s,
		                                 fin.draw));
	// small batches without psf profiles (nothing writes T after the
	// reduction): the gradient step runs inside the reduction's last block
	const bool fold_grad = !recompute && !has_psf_profile(m) && (long long)C * std::max(nrefs, 1) <= 1024;
	GradStepArgs gargs = {dev, nprof, C, nrefs, ref_profile, ref_code, bs.d_ll.as<double>(), invalid, out_ll, out_grad};
	// folded, the step writes logL, the gradient and the queue counters
	// straight into the pinned result buffer (no download afterwards)
	const bool direct_out = fold_grad && bs.h_out_dev && !fit;
	if (direct_out) {
		char *hd = static_cast<char *>(bs.h_out_dev);
		gargs.out_ll = reinterpret_cast<double *>(hd);
		gargs.out_grad = gargs.out_ll + C;
		gargs.ctrl_in = q.counts;
		gargs.ctrl_out = reinterpret_cast<uint32_t *>(hd + (size_t)C * (1 + nrefs) * 8);
		gargs.ctrl_words = CTRL_WORDS;
		if (hmap) {
			// and then the call's sequence number, which the host polls
			gargs.seq_in = reinterpret_cast<const unsigned *>(bs.d_stage.as<char>() + L.seq);
			gargs.seq_out = reinterpret_cast<unsigned *>(hd + out_flag_offset(C, nrefs));
		}
	}
	bs.polled = direct_out && hmap;
	if (!recompute) {
		double *jpart;
		unsigned *jtick;
		PF_TRY(jac_scratch(m, a.dw, a.dh, C * nprof, &jpart, &jtick));
		PF_CUDA(launch_jac_reduce(jac, gconv, gplain, fprof, m->d_prof_batch.as<int>(), C * nprof, a.dw, a.dh,
		                          m->sx / m->fs, m->sy / m->fs, nt, jpart, jtick, bs.d_T.as<double>(), s,
		                          fold_grad ? &gargs : nullptr));
	}
	if (has_psf_profile(m))
		PF_CUDA(launch_psf_adjoint32(dev, m->d_prof_begin.as<int>(), C, nprof, m->d_psf64.as<double>(), m->psf_w,
		                             m->psf_h, m->psf_sx, m->psf_sy, m->sx / m->fs, m->sy / m->fs, a.padx, a.pady,
		                             a.dw, a.dh, gconv, gplain, bs.d_T.as<double>(), s));
	if (!fold_grad)
		PF_CUDA(launch_batch_gradient(dev, nprof, C, ref_profile, ref_code, nrefs, bs.d_T.as<double>(),
		                              bs.d_ll.as<double>(), invalid, out_ll, out_grad, s));
	if (fit && !host_prologue) {
		// LP and d LP / d parm from logL and d logL / d theta
		const int nfit = fit->dev.nfit;
		PF_CUDA(launch_fit_finish(fit->dev, C, bs.d_fit_parm.as<double>(), bs.d_values.as<double>(), out_ll, out_grad,
		                          bs.d_fit_out.as<double>(), s));
		PF_CUDA(cudaMemcpyAsync(bs.h_fit_out.p, bs.d_fit_out.p, (size_t)C * (2 + 2 * nfit) * 8, cudaMemcpyDeviceToHost,
		                        s));
	}
	PF_CUDA(phase_event(m, 3, s));
	char *ho = bs.h_out.as<char>();
	if (!direct_out)
		PF_CUDA(cudaMemcpyAsync(ho, bs.d_out.p, (size_t)C * (1 + nrefs) * 8 + CTRL_WORDS * 4, cudaMemcpyDeviceToHost,
		                        s));
	return PF_OK;
}

// Waits for a chunk's results.  A pipeline that ends by storing the call's
// sequence number after its results (bs.polled) is waited for by polling
// that word in the pinned result buffer: the host sees it a few
// microseconds before the stream reports completion (only the end of the
// last block, which reads nothing more, and the closing timing event
// remain).  The stream is queried now and then, so a launch that fails
// reports its error through the synchronisation below instead of being
// waited for forever.
int wait_chunk(pf_model *m, BatchState &bs, const char *flag_word)
{
	if (bs.polled && flag_word) {
		const volatile unsigned *flag = reinterpret_cast<const volatile unsigned *>(flag_word);
		for (unsigned long spin = 1;; spin++) {
			if (*flag == bs.seq) {
				std::atomic_thread_fence(std::memory_order_acquire);
				return PF_OK;
			}
			if ((spin & 4095) == 0 && cudaStreamQuery(m->stream) != cudaErrorNotReady) break;
		}
	}
	PF_CUDA(cudaStreamSynchronize(m->stream));
	return PF_OK;
}

// B proposals, values[b * nrefs + i] the value of refs[i] in proposal b (null:
// one proposal at the model's current values).  With fit, values holds the
// fitted vectors (fit->host.nfit per proposal) and the results go to fit's
// outputs (LP, d LP / d parm, LL, parm_out) instead of ll_out / grad_out.
int eval_grad_batch(pf_model *m, const pf_param_ref *refs, int nrefs, int B, const double *values, double *ll_out,
                    double *grad_out, const FitRun *fit = nullptr)
{
	PF_TRY(ensure_stream(m));
	Analysis a;
	PF_TRY(analyze(m, a));
	if (!m->has_data) return set_error(PF_E_STATE, "no data: call pf_model_set_data first");
	if (m->data_w != a.ow || m->data_h != a.oh)
		return set_error(PF_E_STATE, "data dimensions differ from the model's output dimensions");
	if (B < 1) return set_error(PF_E_INVALID, "batch size must be positive");
	const int nprof = a.n_profiles;
	if ((long long)B * nprof > 65535 && B > 1) {
		// profile indices of queued cells are 16-bit: chunks keep B*nprof below that
	}
	PF_TRY(upload_psf(m));
	PF_TRY(upload_masks(m, a));
	if (!m->batch) m->batch = new BatchState();
	BatchState &bs = *m->batch;

	// parameter references -> (profile, byte offset, gradient code); the
	// resolution of the previous call is reused while the references and
	// what they resolve against (kind, rescale_flux) are the same
	bool same = (int)bs.refs_key.size() == nrefs && (int)bs.refs_host.size() == 3 * nrefs;
	for (int i = 0; same && i < nrefs; i++) {
		const int pi = refs[i].profile;
		same = pi >= 0 && pi < (int)m->profiles.size() && refs[i].name &&
		       std::get<0>(bs.refs_key[i]) == pi && std::get<1>(bs.refs_key[i]) == m->profiles[pi].kind &&
		       std::get<2>(bs.refs_key[i]) == m->profiles[pi].rescale_flux && std::get<3>(bs.refs_key[i]) == refs[i].name;
	}
	std::vector<int> host_refs;
	if (same) host_refs = bs.refs_host;
	else {
		host_refs.resize(3 * (size_t)nrefs);
		bs.refs_key.clear();
		for (int i = 0; i < nrefs; i++) {
			PF_TRY(check_profile(m, refs[i].profile));
			const ProfileParams &p = m->profiles[refs[i].profile];
			const ParamDesc *d = find_param(p.kind, refs[i].name);
			if (!d || d->type != T_DOUBLE)
				return set_error(PF_E_UNKNOWN_PARAM, std::string("Unknown double parameter: ") + refs[i].name);
			int code = 0;
			PF_TRY(gradient_code(p, refs[i].name, code));
			host_refs[i] = refs[i].profile;
			host_refs[nrefs + i] = (int)d->off;
			host_refs[2 * nrefs + i] = code;
		}
		for (int i = 0; i < nrefs; i++)
			bs.refs_key.emplace_back(refs[i].profile, m->profiles[refs[i].profile].kind,
			                         m->profiles[refs[i].profile].rescale_flux, std::string(refs[i].name));
	}
	std::vector<double> current;
	if (!values) {
		current.resize(nrefs > 0 ? nrefs : 1);
		for (int i = 0; i < nrefs; i++)
			current[i] = *reinterpret_cast<const double *>(
			    reinterpret_cast<const char *>(&m->profiles[host_refs[i]]) + host_refs[nrefs + i]);
		values = current.data();
	}
	if (host_refs != bs.refs_host) {
		PF_CUDA(ensure(bs.d_refs, host_refs.size() * 4 + 4));
		if (nrefs) PF_CUDA(cudaMemcpy(bs.d_refs.p, host_refs.data(), host_refs.size() * 4, cudaMemcpyHostToDevice));
		bs.refs_host = host_refs;
		if (bs.graph) cudaGraphExecDestroy(bs.graph);
		bs.graph = nullptr;
	}

	// chunk size from the memory budget (tangent planes dominate)
	const size_t npix = (size_t)a.dw * a.dh, nout = (size_t)a.ow * a.oh;
	const size_t planes = npix * (size_t)nprof * tangent_stride(m) * 4;
	const bool recompute = m->adjoint_mode == PF_ADJOINT_RECOMPUTE ||
	                       (m->adjoint_mode == PF_ADJOINT_AUTO && planes > (256ull << 20));
	size_t per = npix * (4 * 4 + 8 * 2) + (recompute ? 0 : planes) + nout * (8 + 4) + 4096 +
	             (size_t)a.cw * a.ch * (8 + 4);  // crop window: fine model, fine seed (masks, finesampling)
	if (a.conv && m->conv_kind == CONV_FFT) {
		const size_t spec = (size_t)fft_good_size((int)a.dh + (int)m->psf_h - 1) *
		                    (fft_good_size((int)a.dw + (int)m->psf_w - 1) / 2 + 1);
		per += spec * (sizeof(double2) + sizeof(float2));
	}
	int C = (int)std::min<size_t>((size_t)B, std::max<size_t>(1, BATCH_BUDGET_BYTES / per));
	C = std::min(C, 65535 / std::max(nprof, 1));
	C = std::max(C, 1);

	// buffers for a chunk of C proposals
	PF_CUDA(ensure(m->d_fprof, (size_t)C * nprof * sizeof(FProfile)));
	PF_CUDA(ensure(bs.d_dev, (size_t)C * nprof * sizeof(DevProfile)));
	PF_CUDA(ensure(bs.d_tmpl, nprof * sizeof(ProfileParams)));
	PF_CUDA(ensure(bs.h_tmpl, nprof * sizeof(ProfileParams)));
	// one row of `values` per proposal: model values, or fitted vectors
	const int row = fit ? fit->host.nfit : nrefs;
	PF_CUDA(ensure(bs.d_values, (size_t)C * nrefs * 8 + 8));
	PF_CUDA(ensure(bs.h_values, (size_t)C * std::max(nrefs, row) * 8 + 8));
	if (fit) {
		const size_t fo = (size_t)C * (2 + 2 * (size_t)row) * 8;
		PF_CUDA(ensure(bs.d_fit_parm, (size_t)C * row * 8 + 8));
		PF_CUDA(ensure(bs.d_fit_out, fo));
		PF_CUDA(ensure(bs.h_fit_out, fo));
	}
	PF_CUDA(ensure(bs.d_invalid, (size_t)C * 4));
	PF_CUDA(ensure(bs.d_ll, (size_t)C * 8));
	PF_CUDA(ensure(bs.d_out, (size_t)C * (1 + nrefs) * 8 + CTRL_WORDS * 4));
	PF_CUDA(ensure(bs.d_T, (size_t)C * nprof * NTAN * 8));
	void *out_before = bs.h_out.p;
	PF_CUDA(ensure(bs.h_out, out_flag_offset(C, nrefs) + 256));
	if (bs.h_out.p != out_before || !bs.h_out_dev) {
		if (cudaHostGetDevicePointer(&bs.h_out_dev, bs.h_out.p, 0) != cudaSuccess) {
			cudaGetLastError();
			bs.h_out_dev = nullptr;
		}
	}
	PF_CUDA(ensure(m->d_conv32, npix * C * 4));
	PF_CUDA(ensure(m->d_plain32, npix * C * 4));
	if (!recompute) PF_CUDA(ensure(m->d_jac, npix * tangent_stride(m) * nprof * C * 4));
	PF_CUDA(ensure(m->d_model64, nout * C * 8));
	PF_CUDA(ensure(m->d_wseed, nout * C * 4));
	PF_CUDA(ensure(m->d_gconv, npix * C * 4));
	PF_CUDA(ensure(m->d_gplain, npix * C * 4));
	PF_CUDA(ensure(m->d_partials, (size_t)NPARTS * C * sizeof(double2)));
	if (!(a.conv && m->conv_kind != CONV_NULL)) {
		PF_CUDA(ensure(m->d_conv64, npix * C * 8));
		PF_CUDA(ensure(m->d_plain64, npix * C * 8));
	}
	if (m->prof_begin_n != C * nprof || bs.chunk != C) {
		std::vector<int> begin(C + 1), pb((size_t)C * nprof);
		for (int b = 0; b <= C; b++) begin[b] = b * nprof;
		for (int i = 0; i < C * nprof; i++) pb[i] = i / nprof;
		PF_CUDA(ensure(m->d_prof_begin, (C + 1) * 4));
		PF_CUDA(ensure(m->d_prof_batch, (size_t)C * nprof * 4));
		PF_CUDA(cudaMemcpy(m->d_prof_begin.p, begin.data(), (C + 1) * 4, cudaMemcpyHostToDevice));
		PF_CUDA(cudaMemcpy(m->d_prof_batch.p, pb.data(), (size_t)C * nprof * 4, cudaMemcpyHostToDevice));
		m->prof_begin_n = C * nprof;
		bs.chunk = C;
	}
	std::memcpy(bs.h_tmpl.p, m->profiles.data(), nprof * sizeof(ProfileParams));
	const bool host_prologue = C * nprof <= HOST_PROLOGUE_MAX;
	if (host_prologue) {
		const StageLayout L(C, nprof);
		void *stage_before = bs.h_stage.p;
		PF_CUDA(ensure(bs.h_stage, L.total));
		if (bs.h_stage.p != stage_before || !bs.h_stage_dev) {
			if (cudaHostGetDevicePointer(&bs.h_stage_dev, bs.h_stage.p, 0) != cudaSuccess) {
				cudaGetLastError();
				bs.h_stage_dev = nullptr;
			}
		}
		PF_CUDA(ensure(bs.d_stage, L.total));
	}
	const ModelGeom geom = geometry(m, a);

	char *ho = bs.h_out.as<char>();
	// few-proposal path in fit space: the remake and the chain rule run on the
	// host (the same code as the device kernels)
	std::vector<double> fit_vals, fit_pout;
	if (fit && host_prologue) {
		fit_vals.resize((size_t)C * std::max(nrefs, 1));
		fit_pout.resize((size_t)C * std::max(row, 1));
	}
	for (int b0 = 0; b0 < B; b0 += C) {
		const int n = std::min(C, B - b0);
		// the graph is recorded for full chunks; a short last chunk is padded
		// with copies of its first proposal
		double *hv = bs.h_values.as<double>();
		std::memcpy(hv, values + (size_t)b0 * row, (size_t)n * row * 8);
		for (int b = n; b < C; b++) std::memcpy(hv + (size_t)b * row, values + (size_t)b0 * row, (size_t)row * 8);
		const double *vals = hv;  // model values of the chunk's proposals
		if (fit && host_prologue) {
			for (int b = 0; b < C; b++)
				fit_remake(fit->host, hv + (size_t)b * row, fit_vals.data() + (size_t)b * nrefs,
				           fit_pout.data() + (size_t)b * row);
			vals = fit_vals.data();
		}
		if (host_prologue) {
			const StageLayout L(C, nprof);
			DevProfile *hd = bs.h_stage.as<DevProfile>();
			FProfile *hf = reinterpret_cast<FProfile *>(bs.h_stage.as<char>() + L.f);
			int *hi = reinterpret_cast<int *>(bs.h_stage.as<char>() + L.inv);
			if ((int)m->nq.size() < nprof) m->nq.resize(nprof);
			for (int b = 0; b < C; b++) {
				hi[b] = 0;
				for (int p = 0; p < nprof; p++) {
					ProfileParams pp = m->profiles[p];
					for (int r = 0; r < nrefs; r++)
						if (host_refs[r] == p)
							*reinterpret_cast<double *>(reinterpret_cast<char *>(&pp) + host_refs[nrefs + r]) =
							    vals[(size_t)b * nrefs + r];
					if (!params_valid(pp)) {
						hi[b] = 1;
						pp.kind = PK_NULL;
					}
					derive_profile(pp, geom, hd[b * nprof + p], nullptr, shape_memo(m->nq[p], pp));
					hf[b * nprof + p] = to_fprofile(hd[b * nprof + p], pp);
				}
			}
		}
		bool done = false;
		for (int attempt = 0; attempt < 8 && !done; attempt++) {
			QueueSet q;
			// the pipeline zeroes the counters itself; they sit behind the
			// results so that one copy brings both back
			PF_TRY(prepare_queue(m, a, npix * nprof * C, q, nullptr, nullptr, recompute, false, all_kinds(m)));
			q.counts = reinterpret_cast<uint32_t *>(bs.d_out.as<char>() + (size_t)C * (1 + nrefs) * 8);
			q.overflow = q.counts + MAX_LEVELS;
			q.maxres = q.counts + MAX_LEVELS + 1;
			std::vector<uint64_t> sig = graph_signature(m, a, true, q);
			sig.push_back((uint64_t)C);
			sig.push_back((uint64_t)nrefs);
			sig.push_back((uint64_t)host_prologue);
			sig.push_back((uint64_t)recompute);
			sig.push_back((uint64_t)(uintptr_t)m->d_masks.p);
			sig.push_back((uint64_t)(uintptr_t)bs.h_stage.p);
			for (auto *buf : {&bs.d_tmpl, &bs.d_refs, &bs.d_values, &bs.d_dev, &bs.d_invalid, &bs.d_out, &bs.d_ll,
			                  &bs.d_T, &bs.d_stage})
				sig.push_back((uint64_t)(uintptr_t)buf->p);
			sig.push_back((uint64_t)(uintptr_t)bs.h_out.p);
			sig.push_back((uint64_t)(uintptr_t)bs.h_values.p);
			sig.push_back((uint64_t)(uintptr_t)bs.h_tmpl.p);
			sig.push_back(fit ? 1 + m->fit_version : 0);
			if (fit)
				for (const void *p : std::initializer_list<const void *>{fit->dev.e, bs.d_fit_parm.p, bs.d_fit_out.p,
				                                                         bs.h_fit_out.p})
					sig.push_back((uint64_t)(uintptr_t)p);
			if (host_prologue) {
				// a new sequence number for this launch, and its completion word
				// cleared (pinned memory starts with whatever it held before)
				if (++bs.seq == 0) bs.seq = 1;
				*reinterpret_cast<unsigned *>(bs.h_stage.as<char>() + StageLayout(C, nprof).seq) = bs.seq;
				*reinterpret_cast<volatile unsigned *>(ho + out_flag_offset(C, nrefs)) = 0;
			}
			bool replayed = false;
			if (bs.graph && bs.sig == sig) {
				PF_CUDA(launch_recorded(m, bs.graph));
				note_launches((int)bs.graph_kernels);
				replayed = true;
			}
			else {
				PF_TRY(enqueue_batch_chunk(m, bs, a, C, nrefs, q, host_prologue, recompute, fit));
				m->phases_recorded = true;
			}
			PF_TRY(wait_chunk(m, bs, host_prologue ? ho + out_flag_offset(C, nrefs) : nullptr));
			int retry = 0;
			PF_TRY(check_overflow(m, a, reinterpret_cast<uint32_t *>(ho + (size_t)C * (1 + nrefs) * 8), retry));
			if (retry) {
				PF_CUDA(cudaStreamSynchronize(m->stream));  // (the launch may still be finishing)
				if (bs.graph) cudaGraphExecDestroy(bs.graph);
				bs.graph = nullptr;
				continue;
			}
			done = true;
			finish_timings32(m);
			if (!replayed && m->use_graphs) {
				PF_CUDA(cudaStreamSynchronize(m->stream));
				if (bs.graph) cudaGraphExecDestroy(bs.graph);
				bs.graph = nullptr;
				unsigned long long before = g_launches.load();
				cudaGraph_t graph = nullptr;
				PF_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
				int st = enqueue_batch_chunk(m, bs, a, C, nrefs, q, host_prologue, recompute, fit);
				cudaError_t ce = cudaStreamEndCapture(m->stream, &graph);
				bs.graph_kernels = g_launches.load() - before;
				g_launches -= bs.graph_kernels;
				if (st == PF_OK && ce == cudaSuccess && graph && cudaGraphInstantiate(&bs.graph, graph, 0) == cudaSuccess)
					bs.sig = sig;
				else
					bs.graph = nullptr;
				if (graph) cudaGraphDestroy(graph);
				cudaGetLastError();
			}
		}
		if (!done) return set_error(PF_E_CAPACITY, "subsampling work queue kept overflowing");
		if (fit) {
			const double *ll = reinterpret_cast<const double *>(ho), *g = ll + C;
			for (int b = 0; b < n; b++) {
				double lp, llb, *dlp = fit->grad ? fit->grad + (size_t)(b0 + b) * row : nullptr;
				if (host_prologue) {
					std::vector<double> tmp(dlp ? 0 : row);
					fit_finish_one(fit->host, hv + (size_t)b * row, vals + (size_t)b * nrefs, ll[b], g + (size_t)b * nrefs,
					               &lp, dlp ? dlp : tmp.data(), &llb);
					if (fit->parm_out)
						std::memcpy(fit->parm_out + (size_t)(b0 + b) * row, fit_pout.data() + (size_t)b * row,
						            (size_t)row * 8);
				}
				else {
					const double *fo = bs.h_fit_out.as<double>();
					lp = fo[b];
					llb = fo[(size_t)C * (1 + row) + b];
					if (dlp) std::memcpy(dlp, fo + C + (size_t)b * row, (size_t)row * 8);
					if (fit->parm_out)
						std::memcpy(fit->parm_out + (size_t)(b0 + b) * row, fo + (size_t)C * (2 + row) + (size_t)b * row,
						            (size_t)row * 8);
				}
				fit->lp[b0 + b] = lp;
				if (fit->ll) fit->ll[b0 + b] = llb;
			}
			continue;
		}
		if (ll_out) std::memcpy(ll_out + b0, ho, (size_t)n * 8);
		if (grad_out) std::memcpy(grad_out + (size_t)b0 * nrefs, ho + (size_t)C * 8, (size_t)n * nrefs * 8);
	}
	return PF_OK;
}

// Which tangent combination gives d logL / d(name) for profile p (GradCode),
// or an error for parameters without an adjoint.
int gradient_code(const ProfileParams &p, const char *name, int &code)
{
	if (p.kind == PK_PSF) {  // point source: its centre and magnitude
		if (!std::strcmp(name, "xcen")) code = G_XCEN;
		else if (!std::strcmp(name, "ycen")) code = G_YCEN;
		else if (!std::strcmp(name, "mag")) code = G_MAG;
		else return set_error(PF_E_INVALID, std::string("no gradient with respect to ") + name);
		return PF_OK;
	}
	if (!is_radial_kind(p.kind))
		return set_error(PF_E_INVALID, std::string("no gradient for parameters of ") + kind_name(p.kind) + " profiles");
	if (p.kind == PK_SERSIC && p.rescale_flux)
		return set_error(PF_E_INVALID, "gradients with rescale_flux are not available");
	if (!std::strcmp(name, "xcen")) code = G_XCEN;
	else if (!std::strcmp(name, "ycen")) code = G_YCEN;
	else if (!std::strcmp(name, "mag")) code = G_MAG;
	else if (!std::strcmp(name, "ang")) code = G_ANG;
	else if (!std::strcmp(name, "axrat")) code = G_AXRAT;
	else if (!std::strcmp(name, "box")) code = G_BOX;
	else {
		ProfileParams q = p;
		for (int k = 0; k < shape_count(p.kind); k++) {
			const ParamDesc *d = find_param(p.kind, name);
			if (d && reinterpret_cast<char *>(shape_param(q, k)) - reinterpret_cast<char *>(&q) == (ptrdiff_t)d->off) {
				code = G_SHAPE + k;
				return PF_OK;
			}
		}
		return set_error(PF_E_INVALID, std::string("no gradient with respect to ") + name);
	}
	return PF_OK;
}

int check_profile(pf_model *m, int index)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (index < 0 || index >= (int)m->profiles.size()) return set_error(PF_E_INVALID, "profile index out of range");
	return PF_OK;
}

int set_param(pf_model *m, int index, const char *name, PType type, double dv, unsigned uv, int bv)
{
	PF_TRY(check_profile(m, index));
	ProfileParams &p = m->profiles[index];
	const ParamDesc *d = find_param(p.kind, name);
	if (!d || d->type != type) {
		const char *tn = type == T_DOUBLE ? "double" : type == T_UINT ? "unsigned int" : "bool";
		return set_error(PF_E_UNKNOWN_PARAM, std::string("Unknown ") + tn + " parameter in profile " +
		                                         kind_name(p.kind) + ": " + name);
	}
	char *base = reinterpret_cast<char *>(&p) + d->off;
	if (type == T_DOUBLE) *reinterpret_cast<double *>(base) = dv;
	else if (type == T_UINT) *reinterpret_cast<uint32_t *>(base) = uv;
	else *reinterpret_cast<int32_t *>(base) = bv != 0;
	return PF_OK;
}

std::string trim(const std::string &s)
{
	size_t b = s.find_first_not_of(" \t\n"), e = s.find_last_not_of(" \t\n");
	return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
}

}  // namespace

namespace pf {
// Lets the other translation units of the C ABI report through pf_last_error().
int report_error(int code, const char *msg) { return set_error(code, msg); }
}  // namespace pf

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char *pf_last_error(void) { return g_error.c_str(); }

const char *pf_version(void) { return "profit_b200 0.1 (libprofit 1.9.3 API)"; }

unsigned long long pf_kernel_launches(void) { return pf::g_launches.load(); }

int pf_model_create(unsigned width, unsigned height, pf_model **out)
{
	if (!out) return set_error(PF_E_INVALID, "null output pointer");
	int dev = 0;
	PF_CUDA(cudaGetDevice(&dev));
	cudaDeviceProp prop;
	PF_CUDA(cudaGetDeviceProperties(&prop, dev));
	if (prop.major != 10)
		return set_error(PF_E_CUDA, std::string("profit_b200 needs an sm_100 (B200) device, found ") + prop.name);
	pf_model *m = new pf_model();
	m->width = width;
	m->height = height;
	m->device = dev;
	cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
	for (int i = 0; i < 5 && e == cudaSuccess; i++) e = cudaEventCreate(&m->ev[i]);
	if (e != cudaSuccess) {
		delete m;
		return set_error(PF_E_CUDA, std::string("stream/event creation: ") + cudaGetErrorString(e));
	}
	*out = m;
	return PF_OK;
}

int pf_model_destroy(pf_model *m)
{
	if (!m) return PF_OK;
	cudaSetDevice(m->device);
	if (m->stream) cudaStreamSynchronize(m->stream);
	drop_graph(m);
	delete m->batch;
	m->batch = nullptr;
	for (auto &e : m->ev)
		if (e) cudaEventDestroy(e);
	if (m->stream) cudaStreamDestroy(m->stream);
	delete m;
	return PF_OK;
}

int pf_model_add_profile(pf_model *m, const char *name, int *index)
{
	if (!m || !name) return set_error(PF_E_INVALID, "null argument");
	int k = kind_from_name(name);
	if (k < 0) return set_error(PF_E_INVALID, std::string("Unknown profile name: ") + name);
	m->profiles.push_back(default_params(k));
	if (index) *index = (int)m->profiles.size() - 1;
	return PF_OK;
}

int pf_profile_set_double(pf_model *m, int index, const char *name, double value)
{
	return set_param(m, index, name, T_DOUBLE, value, 0, 0);
}

int pf_profile_set_uint(pf_model *m, int index, const char *name, unsigned value)
{
	return set_param(m, index, name, T_UINT, 0, value, 0);
}

int pf_profile_set_bool(pf_model *m, int index, const char *name, int value)
{
	return set_param(m, index, name, T_BOOL, 0, 0, value);
}

int pf_profile_set(pf_model *m, int index, const char *spec)
{
	PF_TRY(check_profile(m, index));
	std::string s(spec ? spec : "");
	size_t eq = s.find('=');
	if (eq == std::string::npos || s.find('=', eq + 1) != std::string::npos)
		return set_error(PF_E_INVALID, "missing = in parameter: " + s);
	std::string name = trim(s.substr(0, eq)), val = trim(s.substr(eq + 1));
	const ParamDesc *d = find_param(m->profiles[index].kind, name.c_str());
	if (!d)
		return set_error(PF_E_UNKNOWN_PARAM, std::string("Profile ") + kind_name(m->profiles[index].kind) +
		                                         " doesn't support parameter " + name +
		                                         ", or parameter has invalid value: " + val);
	char *end = nullptr;
	if (d->type == T_DOUBLE) {
		double v = std::strtod(val.c_str(), &end);
		if (end == val.c_str()) return set_error(PF_E_INVALID, "Parameter " + name + " cannot be parsed as double: " + val);
		return set_param(m, index, name.c_str(), T_DOUBLE, v, 0, 0);
	}
	unsigned long v = std::strtoul(val.c_str(), &end, 10);
	if (end == val.c_str()) return set_error(PF_E_INVALID, "Parameter " + name + " cannot be parsed: " + val);
	return set_param(m, index, name.c_str(), d->type, 0, (unsigned)v, (int)v);
}

int pf_profile_get_double(pf_model *m, int index, const char *name, double *value)
{
	PF_TRY(check_profile(m, index));
	const ParamDesc *d = find_param(m->profiles[index].kind, name);
	if (!d || d->type != T_DOUBLE)
		return set_error(PF_E_UNKNOWN_PARAM, std::string("Unknown double parameter: ") + name);
	*value = *reinterpret_cast<const double *>(reinterpret_cast<const char *>(&m->profiles[index]) + d->off);
	return PF_OK;
}

int pf_model_profile_count(pf_model *m, int *count)
{
	if (!m || !count) return set_error(PF_E_INVALID, "null argument");
	*count = (int)m->profiles.size();
	return PF_OK;
}

int pf_model_clear_profiles(pf_model *m)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->profiles.clear();
	return PF_OK;
}

int pf_model_set_psf(pf_model *m, const double *psf, unsigned width, unsigned height)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (!psf || width == 0 || height == 0) {
		m->psf.clear();
		m->psf_w = m->psf_h = 0;
		m->psf_dirty = true;
	m->psf_version++;
		return PF_OK;
	}
	size_t n = (size_t)width * height;
	m->psf.assign(psf, psf + n);
	// Image::normalize (image.cpp:231-237): divide by the sum when positive
	double sum = 0;
	for (double v : m->psf) sum += v;
	if (sum > 0)
		for (double &v : m->psf) v /= sum;
	m->psf_w = width;
	m->psf_h = height;
	m->psf_dirty = true;
	m->psf_version++;
	return PF_OK;
}

int pf_model_set_magzero(pf_model *m, double magzero)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->magzero = magzero;
	return PF_OK;
}

int pf_model_set_image_pixel_scale(pf_model *m, double sx, double sy)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->sx = sx;
	m->sy = sy;
	return PF_OK;
}

int pf_model_set_psf_pixel_scale(pf_model *m, double sx, double sy)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->psf_sx = sx;
	m->psf_sy = sy;
	return PF_OK;
}

int pf_model_set_finesampling(pf_model *m, unsigned fs)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (fs == 0) return set_error(PF_E_INVALID, "finesampling must be > 0");
	m->fs = fs;
	return PF_OK;
}

int pf_model_set_return_finesampled(pf_model *m, int value)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->return_fine = value != 0;
	return PF_OK;
}

int pf_model_set_mask(pf_model *m, const uint8_t *mask, unsigned width, unsigned height)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (!mask || width == 0 || height == 0) {
		m->mask.clear();
		m->mask_w = m->mask_h = 0;
		return PF_OK;
	}
	m->mask.assign(mask, mask + (size_t)width * height);
	for (auto &v : m->mask) v = v ? 1 : 0;
	m->mask_w = width;
	m->mask_h = height;
	m->mask_version++;
	return PF_OK;
}

int pf_model_set_dimensions(pf_model *m, unsigned width, unsigned height)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->width = width;
	m->height = height;
	return PF_OK;
}

int pf_model_set_dry_run(pf_model *m, int value)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->dry_run = value != 0;
	return PF_OK;
}

int pf_model_set_omp_threads(pf_model *m, unsigned threads)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	(void)threads;
	return PF_OK;
}

int pf_model_set_adjust_mask(pf_model *m, int value)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->adjust_mask = value != 0;
	return PF_OK;
}

int pf_model_set_crop(pf_model *m, int value)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->crop = value != 0;
	return PF_OK;
}

int pf_model_set_convolver(pf_model *m, const char *type)
{
	if (!m || !type) return set_error(PF_E_INVALID, "null argument");
	if (!std::strcmp(type, "brute") || !std::strcmp(type, "brute-old")) m->conv_kind = CONV_BRUTE;
	else if (!std::strcmp(type, "fft")) m->conv_kind = CONV_FFT;
	else if (!std::strcmp(type, "null")) m->conv_kind = CONV_NULL;
	else return set_error(PF_E_INVALID, std::string("Unknown convolver type: ") + type);
	return PF_OK;
}

// profitDataBenchmark's convolver choice (R/profitSetupData.R:95-110):
// profitBenchmark times each convolver on the model as set up and
// profitBenchmarkResultBest (R/profitBenchmark.R:16-38) keeps the fastest.
// Here "brute" and "fft" are timed on the device (CUDA events) over nbench
// evaluations of what a fit evaluates: logL and its adjoint gradient in the
// FP32 form, logL in the FP64 form, the image when no data are set.
int pf_model_benchmark_convolvers(pf_model *m, int nbench, char *best, size_t best_cap, double *ms_brute,
                                  double *ms_fft)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (nbench < 1) return set_error(PF_E_INVALID, "nbench must be positive");
	const int saved = m->conv_kind;
	const int kinds[2] = {CONV_BRUTE, CONV_FFT};
	const char *names[2] = {"brute", "fft"};
	double ms[2] = {-1, -1};
	std::vector<double> image;
	for (int c = 0; c < 2; c++) {
		m->conv_kind = kinds[c];
		double total = 0;
		int st = PF_OK;
		for (int r = 0; r <= nbench && st == PF_OK; r++) {  // r = 0: warm-up (plans, autotuning, graph capture)
			double ll = 0;
			if (m->has_data && m->precision != PF_FP64) st = pf_model_loglike_grad(m, nullptr, 0, &ll, nullptr);
			else if (m->has_data) st = pf_model_loglike(m, &ll);
			else {
				unsigned w = 0, h = 0;
				int ox = 0, oy = 0;
				st = pf_model_drawing_dims(m, &w, &h);
				image.resize((size_t)w * h);
				if (st == PF_OK) st = pf_model_evaluate(m, image.data(), image.size(), &w, &h, &ox, &oy);
			}
			if (st == PF_OK && r > 0) {
				float t[4];
				pf_model_last_timings(m, t, 4);
				total += t[0];
			}
		}
		if (st == PF_OK) ms[c] = total / nbench;
		else if (c == 0) {
			m->conv_kind = saved;
			return st;  // the model itself does not evaluate
		}
	}
	const int pick = (ms[1] >= 0 && ms[1] < ms[0]) ? 1 : 0;
	m->conv_kind = kinds[pick];
	if (ms_brute) *ms_brute = ms[0];
	if (ms_fft) *ms_fft = ms[1];
	if (best && best_cap) {
		std::strncpy(best, names[pick], best_cap - 1);
		best[best_cap - 1] = 0;
	}
	return PF_OK;
}

int pf_model_set_precision(pf_model *m, int precision)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (precision != PF_FP64 && precision != PF_FP32 && precision != PF_FP32_CONV64)
		return set_error(PF_E_INVALID, "unknown precision");
	m->precision = precision;
	return PF_OK;
}

int pf_model_drawing_dims(pf_model *m, unsigned *w, unsigned *h)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	Analysis a;
	PF_TRY(analyze(m, a));
	if (w) *w = a.dw;
	if (h) *h = a.dh;
	return PF_OK;
}

int pf_model_evaluate(pf_model *m, double *image, size_t capacity, unsigned *out_w, unsigned *out_h, int *offset_x,
                      int *offset_y)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	Analysis a;
	if (m->dry_run) {
		// model.cpp:279-286: inputs checked, a zeroed drawing-size image returned
		PF_TRY(analyze(m, a));
		size_t n = (size_t)a.dw * a.dh;
		if (image) {
			if (capacity < n) return set_error(PF_E_BUFFER, "output buffer too small");
			std::memset(image, 0, n * 8);
		}
		if (out_w) *out_w = a.dw;
		if (out_h) *out_h = a.dh;
		if (offset_x) *offset_x = 0;
		if (offset_y) *offset_y = 0;
		return PF_OK;
	}
	if (m->precision == PF_FP64) {
		PF_TRY(evaluate64(m, a));
		size_t n = (size_t)a.ow * a.oh;
		if (image) {
			if (capacity < n) return set_error(PF_E_BUFFER, "output buffer too small");
			PF_CUDA(cudaMemcpy(image, m->d_model64.p, n * 8, cudaMemcpyDeviceToHost));
		}
	}
	else {
		PF_TRY(evaluate32(m, a, false, nullptr));
		size_t n = (size_t)a.ow * a.oh;
		if (image) {
			if (capacity < n) return set_error(PF_E_BUFFER, "output buffer too small");
			PF_CUDA(cudaMemcpy(image, m->d_model64.p, n * 8, cudaMemcpyDeviceToHost));
		}
	}
	if (out_w) *out_w = a.ow;
	if (out_h) *out_h = a.oh;
	if (offset_x) *offset_x = 0;
	if (offset_y) *offset_y = 0;
	return PF_OK;
}

int pf_model_set_data(pf_model *m, const double *image, const double *sigma, const uint8_t *region, unsigned width,
                      unsigned height)
{
	if (!m || !image || !sigma) return set_error(PF_E_INVALID, "null argument");
	PF_TRY(ensure_stream(m));
	size_t n = (size_t)width * height;
	PF_CUDA(ensure(m->d_data, n * 8));
	PF_CUDA(ensure(m->d_sigma, n * 8));
	PF_CUDA(cudaMemcpy(m->d_data.p, image, n * 8, cudaMemcpyHostToDevice));
	PF_CUDA(cudaMemcpy(m->d_sigma.p, sigma, n * 8, cudaMemcpyHostToDevice));
	m->has_region = region != nullptr;
	if (region) {
		PF_CUDA(ensure(m->d_region, n));
		PF_CUDA(cudaMemcpy(m->d_region.p, region, n, cudaMemcpyHostToDevice));
	}
	m->data_w = width;
	m->data_h = height;
	m->has_data = true;
	return PF_OK;
}

int pf_model_loglike(pf_model *m, double *loglike)
{
	if (!m || !loglike) return set_error(PF_E_INVALID, "null argument");
	if (!m->has_data) return set_error(PF_E_STATE, "no data: call pf_model_set_data first");
	Analysis a;
	if (m->precision == PF_FP64) {
		PF_TRY(evaluate64(m, a));
		if (m->data_w != a.ow || m->data_h != a.oh)
			return set_error(PF_E_STATE, "data dimensions differ from the model's output dimensions");
		PF_CUDA(ensure(m->d_results, 64));
		PF_TRY(enqueue_like(m, m->d_model64.as<double>(), (int)(a.ow * a.oh), 1, m->d_results.as<double>(), nullptr,
		                    m->stream));
		PF_CUDA(cudaMemcpyAsync(loglike, m->d_results.p, 8, cudaMemcpyDeviceToHost, m->stream));
		PF_CUDA(cudaStreamSynchronize(m->stream));
		return PF_OK;
	}
	std::vector<double> res;
	PF_TRY(evaluate32(m, a, false, &res));
	*loglike = res[ResultLayout::LL];
	return PF_OK;
}

int pf_model_set_parameters(pf_model *m, const pf_param_ref *params, int n_params, const double *values)
{
	if (!m || (n_params > 0 && (!params || !values))) return set_error(PF_E_INVALID, "null argument");
	for (int i = 0; i < n_params; i++) PF_TRY(set_param(m, params[i].profile, params[i].name, T_DOUBLE, values[i], 0, 0));
	return PF_OK;
}

int pf_model_loglike_grad(pf_model *m, const pf_param_ref *params, int n_params, double *loglike, double *grad)
{
	if (!m || (n_params > 0 && (!params || !grad))) return set_error(PF_E_INVALID, "null argument");
	if (!m->has_data) return set_error(PF_E_STATE, "no data: call pf_model_set_data first");
	// the current parameter values form a batch of one proposal (values
	// null: read from the profiles)
	double ll = 0;
	PF_TRY(eval_grad_batch(m, params, n_params, 1, nullptr, &ll, grad));
	if (!std::isfinite(ll)) return set_error(PF_E_INVALID, "invalid profile parameters");
	if (loglike) *loglike = ll;
	return PF_OK;
}

int pf_model_loglike_grad_batch(pf_model *m, const pf_param_ref *params, int n_params, int batch,
                                const double *values, double *loglike, double *grad)
{
	if (!m || batch < 1 || (n_params > 0 && (!params || !values)) || !loglike)
		return set_error(PF_E_INVALID, "null argument or empty batch");
	if (!m->has_data) return set_error(PF_E_STATE, "no data: call pf_model_set_data first");
	std::vector<double> scratch;
	if (!grad && n_params > 0) {
		scratch.resize((size_t)batch * n_params);
		grad = scratch.data();
	}
	return eval_grad_batch(m, params, n_params, batch, values, loglike, grad);
}

// ProFit's fit space (profitRemakeModellist, R/profitRemakeModelList.R:27-166;
// profitMakePriors, R/profitUtility.R:124-176), fitspace.cuh.
int pf_model_set_fit_space(pf_model *m, int n, const pf_param_ref *params, const double *init, const int *tofit,
                           const int *tolog, const double *lower, const double *upper, const double *offset,
                           const double *prior_sigma, const double *prior_mean, const int *prior_tolog,
                           const int *prior_on)
{
	if (!m || n < 1 || !params || !init || !tofit) return set_error(PF_E_INVALID, "null argument or no entries");
	PF_TRY(ensure_stream(m));
	FitOffset off{0.0, 0.0, 0.0, 1.0};
	if (offset) {
		if (!std::isfinite(offset[0]) || !std::isfinite(offset[1]))
			return set_error(PF_E_INVALID, "offset x and y must be finite");
		off.x = offset[0];
		off.y = offset[1];
		off.ang = std::isnan(offset[2]) ? 0.0 : offset[2];
		off.size = std::isnan(offset[3]) ? 1.0 : offset[3];
	}
	std::vector<FitEntry> E((size_t)n);
	std::vector<std::pair<int, std::string>> refs;
	int nfit = 0;
	for (int i = 0; i < n; i++) {
		const int pi = params[i].profile;
		const char *name = params[i].name;
		if (!name) return set_error(PF_E_INVALID, "null parameter name");
		PF_TRY(check_profile(m, pi));
		const ParamDesc *d = find_param(m->profiles[pi].kind, name);
		if (!d || d->type != T_DOUBLE)
			return set_error(PF_E_UNKNOWN_PARAM, std::string("Unknown double parameter: ") + name);
		FitEntry e;
		std::memset(&e, 0, sizeof e);
		e.fit = tofit[i] > 0 ? FIT_FREE : tofit[i] < 0 ? FIT_TIED : FIT_FIXED;
		if (i == 0 && e.fit == FIT_TIED)
			return set_error(PF_E_INVALID, "the first entry cannot take its value from the entry before it");
		// R unlogs the entries that are both tolog and fitted (tounlogIDs)
		e.tolog = tolog && tolog[i] && e.fit == FIT_FREE;
		e.fit_index = e.fit == FIT_FREE ? nfit++ : -1;
		e.ref_index = -1;
		if (e.fit != FIT_FIXED) {
			int code = 0;
			PF_TRY(gradient_code(m->profiles[pi], name, code));
			e.ref_index = (int)refs.size();
			refs.emplace_back(pi, std::string(name));
		}
		if (offset) {
			const std::string nm(name);
			if (nm == "xcen") e.offset_bits = OFS_X | OFS_SIZE;
			else if (nm == "ycen") e.offset_bits = OFS_Y | OFS_SIZE;
			else if (nm == "ang") e.offset_bits = OFS_ANG;
			else if (nm == "re" || nm == "fwhm" || nm == "rb" || nm == "rout" || nm == "rc" || nm == "rt")
				e.offset_bits = OFS_SIZE;
		}
		const double lo = lower ? lower[i] : NAN, hi = upper ? upper[i] : NAN;
		e.limited = !(std::isnan(lo) && std::isnan(hi));
		e.lo = std::isnan(lo) ? -INFINITY : lo;
		e.hi = std::isnan(hi) ? INFINITY : hi;
		e.init = init[i];
		if (prior_sigma) {
			const double sg = prior_sigma[i];
			if (!(sg > 0)) return set_error(PF_E_INVALID, "prior sigmas must be positive (inf: flat)");
			const bool on = prior_on ? prior_on[i] != 0 : true;
			e.prior = on && std::isfinite(sg);
			e.prior_sigma = sg;
			e.prior_mean = prior_mean ? prior_mean[i] : init[i];
			e.prior_tolog = prior_tolog ? prior_tolog[i] != 0 : (tolog && tolog[i]);
		}
		E[i] = e;
	}
	if (nfit == 0) return set_error(PF_E_INVALID, "no fitted entry (tofit = 1)");
	// fixed entries do not move with parm: their model value (offsets and
	// clamp applied to init) goes on the profile once
	for (int i = 0; i < n; i++)
		if (E[i].fit == FIT_FIXED)
			PF_TRY(set_param(m, params[i].profile, params[i].name, T_DOUBLE, fit_clamp(E[i], fit_pre_value(E[i], off, nullptr)),
			                 0, 0));
	PF_CUDA(ensure(m->d_fit_entries, E.size() * sizeof(FitEntry)));
	PF_CUDA(cudaMemcpy(m->d_fit_entries.p, E.data(), E.size() * sizeof(FitEntry), cudaMemcpyHostToDevice));
	m->fit_entries = std::move(E);
	m->fit_refs = std::move(refs);
	m->fit_off = off;
	m->fit_nfit = nfit;
	m->fit_version++;
	return PF_OK;
}

int pf_model_fit_size(pf_model *m, int *n_fit, int *n_entries)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (n_fit) *n_fit = m->fit_nfit;
	if (n_entries) *n_entries = (int)m->fit_entries.size();
	return PF_OK;
}

int pf_model_lp_grad_batch(pf_model *m, int batch, const double *parm, double *lp, double *grad, double *parm_out,
                           double *loglike)
{
	if (!m || batch < 1 || !parm || !lp) return set_error(PF_E_INVALID, "null argument or empty batch");
	if (m->fit_entries.empty()) return set_error(PF_E_STATE, "no fit space: call pf_model_set_fit_space first");
	if (!m->has_data) return set_error(PF_E_STATE, "no data: call pf_model_set_data first");
	const int nrefs = (int)m->fit_refs.size();
	std::vector<pf_param_ref> refs((size_t)nrefs);
	for (int i = 0; i < nrefs; i++) refs[i] = pf_param_ref{m->fit_refs[i].first, m->fit_refs[i].second.c_str()};
	FitRun fr;
	fr.host = FitSpaceView{m->fit_entries.data(), (int)m->fit_entries.size(), m->fit_nfit, nrefs, m->fit_off};
	fr.dev = fr.host;
	fr.dev.e = m->d_fit_entries.as<FitEntry>();
	fr.lp = lp;
	fr.grad = grad;
	fr.parm_out = parm_out;
	fr.ll = loglike;
	return eval_grad_batch(m, refs.data(), nrefs, batch, parm, nullptr, nullptr, &fr);
}

int pf_model_loglike_grad_fd(pf_model *m, const pf_param_ref *params, int n_params, double rel_step, double *loglike,
                             double *grad)
{
	if (!m || (n_params > 0 && (!params || !grad))) return set_error(PF_E_INVALID, "null argument");
	if (!m->has_data) return set_error(PF_E_STATE, "no data: call pf_model_set_data first");
	if (!(rel_step > 0)) return set_error(PF_E_INVALID, "rel_step must be positive");
	PF_TRY(ensure_stream(m));
	Analysis a;
	PF_TRY(analyze(m, a));
	if (m->data_w != a.ow || m->data_h != a.oh)
		return set_error(PF_E_STATE, "data dimensions differ from the model's output dimensions");
	PF_TRY(upload_psf(m));
	const int n_eval = 2 * n_params + 1;
	std::vector<double> steps(n_params);
	// parameter sets: base, then (+h, -h) per parameter
	std::vector<std::vector<ProfileParams>> sets(n_eval, m->profiles);
	for (int i = 0; i < n_params; i++) {
		PF_TRY(check_profile(m, params[i].profile));
		const ParamDesc *d = find_param(m->profiles[params[i].profile].kind, params[i].name);
		if (!d || d->type != T_DOUBLE)
			return set_error(PF_E_UNKNOWN_PARAM, std::string("Unknown double parameter: ") + params[i].name);
		double v = *reinterpret_cast<const double *>(reinterpret_cast<const char *>(&m->profiles[params[i].profile]) +
		                                             d->off);
		double h = rel_step * std::max(std::fabs(v), 1.0);
		steps[i] = h;
		for (int sgn = 0; sgn < 2; sgn++) {
			auto &ps = sets[1 + 2 * i + sgn][params[i].profile];
			*reinterpret_cast<double *>(reinterpret_cast<char *>(&ps) + d->off) = sgn == 0 ? v + h : v - h;
			if (const char *err = validate_profile(ps, !m->psf.empty()))
				return set_error(PF_E_INVALID, std::string("finite-difference step leaves the valid range: ") + err);
		}
	}
	size_t npix = (size_t)a.dw * a.dh;
	PF_CUDA(ensure(m->d_partials, NPARTS * sizeof(double2)));
	PF_CUDA(ensure(m->d_results, (size_t)n_eval * 8));
	PF_CUDA(ensure(m->h_results, (size_t)n_eval * 8 + CTRL_WORDS * 4 * n_eval));
	for (int attempt = 0; attempt < 8; attempt++) {
		PF_CUDA(record_event(m->ev[0], m->stream));
		for (int e = 0; e < n_eval; e++) PF_TRY(derive_and_upload(m, a, sets[e], e, n_eval, false));
		uint32_t *hctrl = reinterpret_cast<uint32_t *>(m->h_results.as<char>() + (size_t)n_eval * 8);
		for (int e = 0; e < n_eval; e++) {
			QueueSet q;
			PF_TRY(prepare_queue(m, a, npix * a.n_profiles, q, nullptr, nullptr));
			PF_TRY(run_plain64(m, a, m->d_prof.as<DevProfile>() + (size_t)e * a.n_profiles, q));
			PF_TRY(enqueue_like(m, m->d_model64.as<double>(), (int)(a.ow * a.oh), 1, m->d_results.as<double>() + e,
			                    nullptr, m->stream));
			PF_CUDA(cudaMemcpyAsync(hctrl + (size_t)e * CTRL_WORDS, m->d_ctrl.p, CTRL_WORDS * 4,
			                        cudaMemcpyDeviceToHost, m->stream));
		}
		PF_CUDA(cudaMemcpyAsync(m->h_results.p, m->d_results.p, (size_t)n_eval * 8, cudaMemcpyDeviceToHost,
		                        m->stream));
		PF_CUDA(record_event(m->ev[3], m->stream));
		PF_CUDA(cudaStreamSynchronize(m->stream));
		int retry = 0;
		for (int e = 0; e < n_eval; e++) {
			int r = 0;
			PF_TRY(check_overflow(m, a, hctrl + (size_t)e * CTRL_WORDS, r));
			retry |= r;
		}
		if (retry) continue;
		const double *ll = m->h_results.as<double>();
		if (loglike) *loglike = ll[0];
		for (int i = 0; i < n_params; i++) grad[i] = (ll[1 + 2 * i] - ll[2 + 2 * i]) / (2 * steps[i]);
		m->timings_lazy = false;
		cudaEventElapsedTime(&m->timings[0], m->ev[0], m->ev[3]);
		cudaGetLastError();
		return PF_OK;
	}
	return set_error(PF_E_CAPACITY, "subsampling work queue kept overflowing");
}

int pf_model_set_likelihood(pf_model *m, const char *name)
{
	if (!m || !name) return set_error(PF_E_INVALID, "null argument");
	std::string f(name);
	for (auto &ch : f) ch = (char)std::tolower((unsigned char)ch);
	int kind;
	if (f == "norm" || f == "normal") kind = LIKE_NORM;
	else if (f == "chisq" || f == "chi-sq") kind = LIKE_CHISQ;
	else if (f == "t" || f == "student" || f == "student-t") kind = LIKE_T;
	else if (f == "pois" || f == "poisson" || f == "cash" || f == "c") kind = LIKE_POIS;
	else if (f == "st" || f == "skewt" || f == "skew-t")
		return set_error(PF_E_INVALID, "the skew-t likelihood (LaplacesDemon fit of its parameters) is not available");
	else
		return set_error(PF_E_INVALID, std::string("Error: unknown likelihood function: '") + f + "'");
	if (kind != m->like_kind) drop_graph(m);
	m->like_kind = kind;
	return PF_OK;
}

int pf_model_set_adjoint_mode(pf_model *m, int mode)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	if (mode != PF_ADJOINT_AUTO && mode != PF_ADJOINT_STORE && mode != PF_ADJOINT_RECOMPUTE)
		return set_error(PF_E_INVALID, "unknown adjoint mode");
	m->adjoint_mode = mode;
	return PF_OK;
}

int pf_model_set_phase_timing(pf_model *m, int on)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->phase_timing = on != 0;
	return PF_OK;
}

int pf_model_set_debug(pf_model *m, int value)
{
	if (!m) return set_error(PF_E_INVALID, "null model");
	m->debug = value != 0;
	return PF_OK;
}

int pf_model_decisions(pf_model *m, int profile, int32_t *out, size_t capacity)
{
	PF_TRY(check_profile(m, profile));
	if (m->decisions.empty()) return set_error(PF_E_STATE, "no decisions recorded: enable debug and evaluate");
	if (capacity < m->dec_npix) return set_error(PF_E_BUFFER, "output buffer too small");
	std::memcpy(out, m->decisions.data() + (size_t)profile * m->dec_npix, (size_t)m->dec_npix * 4);
	return PF_OK;
}

int pf_model_level_counts(pf_model *m, int profile, int64_t *out, int max_levels, int *n_levels)
{
	PF_TRY(check_profile(m, profile));
	if (m->level_counts.empty()) return set_error(PF_E_STATE, "no counters recorded: enable debug and evaluate");
	int n = 0;
	for (int l = 0; l < MAX_LEVELS; l++) {
		unsigned long long c = m->level_counts[(size_t)profile * MAX_LEVELS + l];
		if (l < max_levels) out[l] = (int64_t)c;
		if (c) n = l + 1;
	}
	if (n_levels) *n_levels = n;
	return PF_OK;
}

int pf_model_evaluation_counts(pf_model *m, int profile, int64_t *out, int max_levels, int64_t *total)
{
	PF_TRY(check_profile(m, profile));
	if (m->evals.empty()) return set_error(PF_E_STATE, "no counters recorded: enable debug and evaluate");
	const unsigned long long *e = m->evals.data() + (size_t)profile * (1 + MAX_LEVELS);
	unsigned long long sum = 0;
	for (int l = 0; l < 1 + MAX_LEVELS; l++) {
		if (out && l < max_levels) out[l] = (int64_t)e[l];
		sum += e[l];
	}
	if (total) *total = (int64_t)sum;
	return PF_OK;
}

int pf_model_last_timings(pf_model *m, float *ms, int n)
{
	if (!m || !ms) return set_error(PF_E_INVALID, "null argument");
	if (m->timings_lazy) resolve_timings32(m);
	for (int i = 0; i < n && i < 4; i++) ms[i] = m->timings[i];
	return PF_OK;
}

}  // extern "C"

// ===========================================================================
// Catalogue batches: many galaxies, each with its own image size, PSF, data
// and profiles, evaluated together.  Galaxies are grouped into buckets of one
// canvas size and one PSF size; inside a bucket each galaxy sits at the
// top-left of the canvas, its extra pixels carry zero weight (region mask),
// and its own PSF and data are picked by batch index.  A larger canvas leaves
// the cropped model of a galaxy unchanged: the PSF reaches only psf/2 pixels
// beyond the image, and that border is drawn for every galaxy.
//
// One evaluation: one FP64 prologue launch for every profile of the
// catalogue, then every chunk's pipeline back to back on one stream (scratch
// and queue sized up front for the largest chunk), one synchronisation, and
// a re-run of any chunk whose subsampling queue overflowed.
// ===========================================================================

namespace {

struct CatGalaxy {
	unsigned w = 0, h = 0, pw = 0, ph = 0;
	std::vector<double> data, sigma, psf;  // psf normalised
	std::vector<ProfileParams> profiles;
};

// A typed view of part of a larger buffer.
struct Span {
	void *p = nullptr;
	template <class T>
	T *as() const
	{
		return static_cast<T *>(p);
	}
};

// One launch group: galaxies of one bucket, static inputs resident.
struct CatChunk {
	unsigned W = 0, H = 0, pw = 0, ph = 0;
	std::vector<int> members;           // galaxy indices
	std::vector<int> member_grad_off;   // offset of each member's gradient in the chunk's buffer
	int p0 = 0, nprof = 0, ngrad = 0, levels = 1, nt = NTAN_GEOM + 3, cusps = 0;
	int lane = 0;  // the engine (stream and scratch) its recorded pipeline runs on
	// convolutions through FP64 FFTs (each member's PSF spectrum in kspec)
	// instead of the brute-force kernels: the faster of the two, timed at build
	bool fft = false;
	FftConv<double> fc;
	Span kspec;  // in pf_catalogue::spectra
	bool ak = false;
	bool plain = false;  // a profile drawn without convolution (reads the seed of the plain image)
	// slices of the catalogue's shared device and pinned host arenas
	Span data, sigma, region, psf32, psfrev32;
	Span prof_begin, prof_batch, grad_off, T, ll, grad;
	Span extent;  // per member, the drawing its outputs read (int2: own width, height + the PSF padding)
	Span h_ll, h_grad, h_ctrl;
	size_t npix() const { return (size_t)(W + 2 * (pw / 2)) * (H + 2 * (ph / 2)); }
	size_t nout() const { return (size_t)W * H; }
};

constexpr size_t CAT_BUDGET_BYTES = 6ull << 30;
// PSF spectra of the chunks that convolve through FFTs, all chunks together
constexpr size_t CAT_SPECTRA_BYTES = 16ull << 30;
enum CatConv : int { CAT_CONV_AUTO = 0, CAT_CONV_BRUTE, CAT_CONV_FFT };

// PF_CATALOGUE_LOG=1: the host time of each step of a call that builds or
// records, on stderr.
bool cat_log_on()
{
	static const bool on = [] {
		const char *v = getenv("PF_CATALOGUE_LOG");
		return v && v[0] == '1';
	}();
	return on;
}

double cat_now()
{
	return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
// Engines whose streams run chunks side by side in the recorded call: the
// small kernels of one chunk (the cusp levels, the likelihood, the tails of
// the waves) leave SMs idle that another chunk's kernels fill.  (10,000
// galaxies on one B200: 222.5 ms per call with 4, 219.7 with 6, 218.9 with 8,
// whose first call took longer.)
constexpr int CAT_LANES = 6;
constexpr unsigned CAT_SIDE_STEP = 64;

}  // namespace

struct pf_catalogue {
	std::vector<CatGalaxy> gal;
	double magzero = 0;
	pf_model *engine = nullptr;  // stream, scratch buffers, queue capacities
	std::vector<pf_model *> lanes;  // lanes[0] is engine; each with its own stream and scratch
	std::vector<size_t> lane_qpix;  // drawing pixels of each lane's largest chunk (queue sizing)
	int max_levels = 1;
	cudaEvent_t fork = nullptr;
	std::vector<cudaEvent_t> joins;
	bool built = false;
	std::vector<std::unique_ptr<CatChunk>> chunks;
	DevBuf params, pad, dev, fprof;  // every profile of the catalogue, chunk after chunk
	DevBuf lum;                       // LUM_SLOTS luminosity evaluations per profile (prologue scratch)
	DevBuf arena;                     // every chunk's index tables, tangent sums, logL and gradient
	DevBuf canvases;                  // every chunk's data, sigma, region and PSF images
	DevBuf spectra, spectra_trial;    // PSF spectra of the FFT chunks; one chunk's, while timing
	HostBuf h_arena;                  // every chunk's logL, gradient and queue control words
	int nprof = 0;
	std::vector<int> grad_off;
	int grad_total = 0;
	bool params_dirty = false;  // set_values changed profiles since the last upload
	int conv_mode = CAT_CONV_AUTO;  // how chunks pick their convolver (pf_catalogue_set_convolver)
	float last_ms = 0;
	cudaEvent_t ev[2] = {};
	// the whole call (prologue and every chunk) captured once and replayed
	// while the queue capacities it was captured with hold
	cudaGraphExec_t graph = nullptr;
	std::vector<uint32_t> graph_caps;
	unsigned long long graph_kernels = 0;
};

namespace {

// Parameter k of a catalogue profile in the order of its gradient: xcen,
// ycen, mag, ang, axrat, box, then the kind's shape parameters.
double *cat_value_slot(ProfileParams &p, int k)
{
	switch (k) {
	case 0: return &p.xcen;
	case 1: return &p.ycen;
	case 2: return &p.mag;
	case 3: return &p.ang;
	case 4: return &p.axrat;
	case 5: return &p.box;
	default: return shape_param(p, k - 6);
	}
}

int cat_set_param(ProfileParams &p, const char *name, double value)
{
	const ParamDesc *d = find_param(p.kind, name);
	if (!d)
		return set_error(PF_E_UNKNOWN_PARAM, std::string("Unknown parameter in profile ") + kind_name(p.kind) + ": " +
		                                         name);
	char *base = reinterpret_cast<char *>(&p) + d->off;
	if (d->type == T_DOUBLE) *reinterpret_cast<double *>(base) = value;
	else if (d->type == T_UINT) *reinterpret_cast<uint32_t *>(base) = (uint32_t)value;
	else *reinterpret_cast<int32_t *>(base) = value != 0;
	return PF_OK;
}

Analysis cat_analysis(const CatChunk &ch)
{
	Analysis a;
	a.conv = true;
	a.padx = ch.pw / 2;
	a.pady = ch.ph / 2;
	a.cw = ch.W;
	a.ch = ch.H;
	a.dw = ch.W + 2 * a.padx;
	a.dh = ch.H + 2 * a.pady;
	a.ow = ch.W;
	a.oh = ch.H;
	a.levels = ch.levels;
	a.n_profiles = ch.nprof;
	return a;
}

// The chunk's forward convolution: the drawing (FP32, batch of C) into the
// FP64 model image on the crop window, plus the unconvolved drawing.  Brute
// force: out(x) = sum_i conv(x + i) psf(pw - 1 - i).  FFT: the same sum is
// the linear convolution read at offset pw - 1; on a grid of at least the
// drawing's size nothing it reads wraps around.
int cat_conv_forward(pf_model *m, CatChunk &ch, const Analysis &a, bool fft, const float *conv, const float *plain,
                     double *model64, cudaStream_t s)
{
	const int C = (int)ch.members.size();
	const size_t npix = ch.npix(), nout = ch.nout();
	if (fft) {
		PF_CUDA(ch.fc.convolve<float, double, float>(conv, a.dw, a.dh, 0, 0, ch.kspec.as<double2>(), false,
		                                             m->d_fftwork64.as<double2>(), (int)ch.pw - 1, (int)ch.ph - 1,
		                                             model64, a.cw, a.ch, plain, a.dw, a.padx, a.pady, C, npix, nout,
		                                             npix, s, ch.fc.spectrum_elems()));
		note_launches(3);
		return PF_OK;
	}
	const size_t sb = conv32_scratch_bytes(a.cw, a.ch, C);
	PF_CUDA(launch_conv32_to64(conv, a.dw, a.dh, 0, 0, ch.psfrev32.as<float>(), ch.pw, ch.ph, model64, a.cw, a.ch,
	                           plain, a.dw, a.padx, a.pady, C, (int)npix, (int)nout,
	                           sb ? m->d_convsplit.as<double>() : nullptr, sb, (int)(ch.pw * ch.ph), s));
	return PF_OK;
}

// Its adjoint: dlogL/dmodel (wseed, crop window) to dlogL/d(drawing pixel),
// g(U) = sum_i w(U + 1 - pw + i) psf(i); through FFTs, the correlation with
// the seed placed at pw - 1 (on a grid of at least the drawing's size, what
// wraps around lands on the zeros below that offset).
int cat_conv_adjoint(pf_model *m, CatChunk &ch, const Analysis &a, bool fft, const float *wseed, float *gconv,
                     cudaStream_t s)
{
	const int C = (int)ch.members.size();
	const size_t npix = ch.npix(), nout = ch.nout();
	if (fft) {
		PF_CUDA(ch.fc.convolve<float, float, float>(wseed, a.ow, a.oh, (int)ch.pw - 1, (int)ch.ph - 1,
		                                            ch.kspec.as<double2>(), true, m->d_fftwork64.as<double2>(), 0, 0,
		                                            gconv, a.dw, a.dh, nullptr, 0, 0, 0, C, nout, npix, 0, s,
		                                            ch.fc.spectrum_elems()));
		note_launches(3);
		return PF_OK;
	}
	const size_t sb = conv32_scratch_bytes(a.dw, a.dh, C);
	PF_CUDA(launch_conv32(wseed, a.ow, a.oh, 1 - (int)ch.pw, 1 - (int)ch.ph, ch.psf32.as<float>(), ch.pw, ch.ph, gconv,
	                      a.dw, a.dh, nullptr, 0, 0, 0, C, (int)nout, (int)npix,
	                      sb ? m->d_convsplit.as<double>() : nullptr, sb, (int)(ch.pw * ch.ph), s));
	return PF_OK;
}

void release(DevBuf &b)
{
	if (b.p) cudaFree(b.p);
	b.p = nullptr;
	b.bytes = 0;
}

// Each chunk's convolver: brute force, or FP64 FFTs with the members' PSF
// spectra.  Under CAT_CONV_AUTO both are timed on the chunk itself (forward
// and adjoint, after a warm-up run, which also tunes the brute-force tile) on
// lane 0, whose scratch takes every chunk, and the faster is kept; brute
// force is not timed (nor tuned) where the FFTs beat its FLOP count at the
// GPU's FP32 peak.  The timed runs read zeroed drawings and write only
// buffers that every evaluation rewrites.  The trials share one spectrum
// buffer; the chosen chunks' spectra then go into one allocation (a device
// allocation and release per chunk had made this step take 0.1-1 s more,
// varying from run to run).
int cat_pick_convolvers(pf_catalogue *c)
{
	pf_model *m = c->lanes[0];
	cudaStream_t s = m->stream;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	PF_CUDA(cudaEventCreate(&e0));
	PF_CUDA(cudaEventCreate(&e1));
	struct Events {
		cudaEvent_t &a, &b;
		~Events()
		{
			if (a) cudaEventDestroy(a);
			if (b) cudaEventDestroy(b);
		}
	} guard{e0, e1};
	// an upper bound on the GPU's FP32 rate: 128 FMA lanes per SM at the
	// highest SM clock, with a quarter more for safety
	int sms = 0, khz = 0;
	PF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device));
	PF_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, m->device));
	const double fp32_peak = 1.25 * 256.0 * sms * (khz * 1e3);
	double t_alloc = 0, t_fft_trials = 0, t_brute_trials = 0;  // host time, for the timing log

	// the chunks that may convolve through FFTs: their grids and spectra sizes
	std::vector<size_t> need(c->chunks.size(), 0);
	size_t most = 0;
	for (size_t k = 0; k < c->chunks.size(); k++) {
		CatChunk &ch = *c->chunks[k];
		ch.fft = false;
		ch.kspec.p = nullptr;
		if (c->conv_mode == CAT_CONV_BRUTE) continue;
		const Analysis a = cat_analysis(ch);
		const int N = fft_good_size((int)a.dw), M = fft_good_size((int)a.dh);
		if (N > FFT_MAX_LEN || M > FFT_MAX_LEN) continue;
		if (ch.fc.setup(M, N) != cudaSuccess) {
			cudaGetLastError();
			continue;
		}
		need[k] = ch.fc.spectrum_elems() * sizeof(double2) * ch.members.size();
		most = std::max(most, need[k]);
	}
	if (most) {
		const double t0 = cat_now();
		PF_CUDA(ensure(c->spectra_trial, most));
		PF_CUDA(ensure(m->d_fftwork64, most));
		t_alloc += cat_now() - t0;
	}

	size_t spectra = 0;
	std::vector<size_t> work(c->lanes.size(), 0);
	for (size_t k = 0; k < c->chunks.size(); k++) {
		CatChunk &ch = *c->chunks[k];
		if (!need[k] || spectra + need[k] > CAT_SPECTRA_BYTES) continue;
		const int C = (int)ch.members.size();
		bool use = c->conv_mode == CAT_CONV_FFT;
		if (!use) {
			const Analysis a = cat_analysis(ch);
			ch.kspec.p = c->spectra_trial.p;
			PF_CUDA(ch.fc.set_kernels(ch.psf32.as<float>(), (int)ch.pw, (int)ch.ph, (size_t)ch.pw * ch.ph,
			                          ch.kspec.as<double2>(), C, s));
			note_launches(2);
			float *conv = m->d_conv32.as<float>(), *plain = m->d_plain32.as<float>();
			float *wseed = m->d_wseed.as<float>(), *gconv = m->d_gconv.as<float>();
			PF_CUDA(cudaMemsetAsync(conv, 0, ch.npix() * C * 4, s));
			PF_CUDA(cudaMemsetAsync(plain, 0, ch.npix() * C * 4, s));
			PF_CUDA(cudaMemsetAsync(wseed, 0, ch.nout() * C * 4, s));
			auto run = [&](bool fft) -> int {
				PF_TRY(cat_conv_forward(m, ch, a, fft, conv, plain, m->d_model64.as<double>(), s));
				return cat_conv_adjoint(m, ch, a, fft, wseed, gconv, s);
			};
			auto timed = [&](bool fft, float &best) -> int {
				PF_TRY(run(fft));  // warm-up (brute force: tunes the tile for this shape)
				best = 1e30f;
				for (int r = 0; r < 2; r++) {
					PF_CUDA(cudaEventRecord(e0, s));
					PF_TRY(run(fft));
					PF_CUDA(cudaEventRecord(e1, s));
					PF_CUDA(cudaEventSynchronize(e1));
					float ms = 0;
					PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
					best = std::min(best, ms);
					if (ms > 2.0f) break;  // long enough to be timed once
				}
				return PF_OK;
			};
			float t_fft = 0, t_brute = 0;
			double t0 = cat_now();
			PF_TRY(timed(true, t_fft));
			t_fft_trials += cat_now() - t0;
			// brute force cannot beat its multiply-adds at the FP32 peak: an
			// FFT faster than that wins without tuning and timing the tiles
			const double flop = 2.0 * ch.pw * ch.ph * (double)(ch.nout() + ch.npix()) * C;
			if (t_fft * 1e-3 < flop / fp32_peak) {
				use = true;
			}
			else {
				t0 = cat_now();
				PF_TRY(timed(false, t_brute));
				t_brute_trials += cat_now() - t0;
				use = t_fft < t_brute;
			}
			ch.kspec.p = nullptr;
		}
		if (use) {
			ch.fft = true;
			spectra += need[k];
			work[0] = std::max(work[0], need[k]);
			work[ch.lane] = std::max(work[ch.lane], need[k]);
		}
	}

	// the FFT chunks' spectra, one allocation for all of them
	double t0 = cat_now();
	if (spectra) PF_CUDA(ensure(c->spectra, spectra));
	size_t off = 0;
	for (size_t k = 0; k < c->chunks.size(); k++) {
		CatChunk &ch = *c->chunks[k];
		if (!ch.fft) continue;
		ch.kspec.p = c->spectra.as<char>() + off;
		off += need[k];
		PF_CUDA(ch.fc.set_kernels(ch.psf32.as<float>(), (int)ch.pw, (int)ch.ph, (size_t)ch.pw * ch.ph,
		                          ch.kspec.as<double2>(), (int)ch.members.size(), s));
		note_launches(2);
	}
	PF_CUDA(cudaStreamSynchronize(s));
	release(c->spectra_trial);
	for (size_t l = 0; l < c->lanes.size(); l++)
		if (work[l]) PF_CUDA(ensure(c->lanes[l]->d_fftwork64, work[l]));
	t_alloc += cat_now() - t0;
	if (cat_log_on())
		fprintf(stderr,
		        "[profit_b200 catalogue] convolver trials: FFT %.3f s, brute force (with tuning) %.3f s, "
		        "spectra %.3f s\n",
		        t_fft_trials, t_brute_trials, t_alloc);
	return PF_OK;
}

// Groups galaxies into chunks and uploads the static inputs.
int cat_build(pf_catalogue *c)
{
	const double t_build = cat_now();
	// the chunks and their buffers are rebuilt: a recorded call no longer applies
	if (c->graph) cudaGraphExecDestroy(c->graph);
	c->graph = nullptr;
	// gradient layout: per galaxy, per profile (xcen, ycen, mag, ang, axrat, box, shape...)
	c->grad_off.assign(c->gal.size(), 0);
	int total = 0;
	for (size_t g = 0; g < c->gal.size(); g++) {
		c->grad_off[g] = total;
		for (auto &p : c->gal[g].profiles) total += 6 + shape_count(p.kind);
	}
	c->grad_total = total;
	// buckets: canvas side class x PSF size
	std::map<std::tuple<unsigned, unsigned, unsigned>, std::vector<int>> buckets;
	for (size_t g = 0; g < c->gal.size(); g++) {
		const CatGalaxy &G = c->gal[g];
		unsigned side = std::max(G.w, G.h);
		unsigned cls = (side + CAT_SIDE_STEP - 1) / CAT_SIDE_STEP;
		buckets[std::make_tuple(cls, G.pw, G.ph)].push_back((int)g);
	}
	c->chunks.clear();
	for (auto &kv : buckets) {
		const auto &mem = kv.second;
		unsigned W = 0, H = 0;
		for (int g : mem) {
			W = std::max(W, c->gal[g].w);
			H = std::max(H, c->gal[g].h);
		}
		const unsigned pw = std::get<1>(kv.first), ph = std::get<2>(kv.first);
		const size_t npix = (size_t)(W + 2 * (pw / 2)) * (H + 2 * (ph / 2)), nout = (size_t)W * H;
		size_t start = 0;
		while (start < mem.size()) {
			// members of this chunk: scratch within the budget, profile index within 16 bits
			size_t bytes = 0, end = start;
			int np = 0;
			while (end < mem.size()) {
				const int g = mem[end];
				const int gp = (int)c->gal[g].profiles.size();
				const size_t b = npix * (8 + 12) + nout * (8 + 4) + (size_t)gp * NTAN * npix * sizeof(double);
				if (end > start && (bytes + b > CAT_BUDGET_BYTES || np + gp > 60000)) break;
				bytes += b;
				np += gp;
				end++;
			}
			auto ch = std::make_unique<CatChunk>();
			ch->W = W;
			ch->H = H;
			ch->pw = pw;
			ch->ph = ph;
			ch->members.assign(mem.begin() + start, mem.begin() + end);
			start = end;
			c->chunks.push_back(std::move(ch));
		}
	}
	// static inputs: profile records and per-chunk index tables (serial and
	// cheap; the tables go up in one copy into a shared arena), then every
	// chunk's images (below, in parallel)
	std::vector<ProfileParams> params;
	std::vector<int2> pad;
	std::vector<unsigned char> tables;  // the arena's index tables, at their offsets
	size_t dtop = 0, htop = 0;
	auto take = [](size_t &top, size_t bytes) {
		const size_t o = top;
		top += (std::max<size_t>(bytes, 8) + 255) & ~(size_t)255;
		return o;
	};
	auto put = [&](const std::vector<int> &v) {
		const size_t o = take(dtop, v.size() * 4);
		tables.resize(dtop);
		if (!v.empty()) std::memcpy(tables.data() + o, v.data(), v.size() * 4);
		return o;
	};
	struct Slots {
		size_t prof_begin, prof_batch, grad_off, extent, T, ll, grad, h_ll, h_grad, h_ctrl;
	};
	std::vector<Slots> slots(c->chunks.size());
	for (size_t k = 0; k < c->chunks.size(); k++) {
		CatChunk &ch = *c->chunks[k];
		const int C = (int)ch.members.size();
		std::vector<int> prof_begin(C + 1, 0), prof_batch, goff;
		ch.member_grad_off.assign(C, 0);
		ch.p0 = (int)params.size();
		int gtot = 0;
		for (int i = 0; i < C; i++) {
			const CatGalaxy &G = c->gal[ch.members[i]];
			ch.member_grad_off[i] = gtot;
			for (auto &p : G.profiles) {
				params.push_back(p);
				pad.push_back(make_int2((int)(ch.pw / 2), (int)(ch.ph / 2)));
				prof_batch.push_back(i);
				goff.push_back(gtot);
				gtot += 6 + shape_count(p.kind);
				unsigned mr = p.max_recursions;
				// an adjusted Sersic may have its centre cusp (nser > 1) after
				// pf_catalogue_set_values, so the levels are kept for it either way
				if (p.kind == PK_SERSIC && p.adjust) {
					mr = std::max(mr, 10u);
					if (p.nser > 1) ch.cusps++;
				}
				ch.levels = std::max(ch.levels, (int)mr + 1);
				ch.nt = std::max(ch.nt, tangent_count(p.kind));
				if (p.kind != PK_SERSIC && p.kind != PK_MOFFAT) ch.ak = true;
				if (!p.convolve) ch.plain = true;
			}
			prof_begin[i + 1] = (int)params.size() - ch.p0;
		}
		ch.nprof = (int)params.size() - ch.p0;
		ch.ngrad = gtot;
		Slots &sl = slots[k];
		sl.prof_begin = put(prof_begin);
		sl.prof_batch = put(prof_batch);
		sl.grad_off = put(goff);
		std::vector<int> ext(2 * (size_t)C);
		for (int i = 0; i < C; i++) {
			const CatGalaxy &G = c->gal[ch.members[i]];
			ext[2 * i] = (int)(G.w + 2 * (ch.pw / 2));
			ext[2 * i + 1] = (int)(G.h + 2 * (ch.ph / 2));
		}
		sl.extent = put(ext);
		sl.T = take(dtop, (size_t)ch.nprof * NTAN * 8);
		sl.ll = take(dtop, (size_t)C * 8);
		sl.grad = take(dtop, (size_t)std::max(gtot, 1) * 8);
		sl.h_ll = take(htop, (size_t)C * 8);
		sl.h_grad = take(htop, (size_t)std::max(gtot, 1) * 8);
		sl.h_ctrl = take(htop, CTRL_WORDS * 4);
	}
	PF_CUDA(ensure(c->arena, dtop));
	PF_CUDA(cudaMemcpy(c->arena.p, tables.data(), tables.size(), cudaMemcpyHostToDevice));
	PF_CUDA(ensure(c->h_arena, htop));
	// the images of every chunk in one allocation
	size_t ctop = 0;
	std::vector<std::array<size_t, 5>> coff(c->chunks.size());
	for (size_t k = 0; k < c->chunks.size(); k++) {
		const CatChunk &ch = *c->chunks[k];
		const size_t C = ch.members.size(), nout = ch.nout(), nk = (size_t)ch.pw * ch.ph;
		coff[k] = {take(ctop, nout * C * 8), take(ctop, nout * C * 8), take(ctop, nout * C), take(ctop, C * nk * 4),
		           take(ctop, C * nk * 4)};
	}
	PF_CUDA(ensure(c->canvases, ctop));
	for (size_t k = 0; k < c->chunks.size(); k++) {
		CatChunk &ch = *c->chunks[k];
		char *d = c->canvases.as<char>();
		ch.data.p = d + coff[k][0];
		ch.sigma.p = d + coff[k][1];
		ch.region.p = d + coff[k][2];
		ch.psf32.p = d + coff[k][3];
		ch.psfrev32.p = d + coff[k][4];
	}
	for (size_t k = 0; k < c->chunks.size(); k++) {
		CatChunk &ch = *c->chunks[k];
		const Slots &sl = slots[k];
		char *d = c->arena.as<char>(), *h = c->h_arena.as<char>();
		ch.prof_begin.p = d + sl.prof_begin;
		ch.prof_batch.p = d + sl.prof_batch;
		ch.grad_off.p = d + sl.grad_off;
		ch.extent.p = d + sl.extent;
		ch.T.p = d + sl.T;
		ch.ll.p = d + sl.ll;
		ch.grad.p = d + sl.grad;
		ch.h_ll.p = h + sl.h_ll;
		ch.h_grad.p = h + sl.h_grad;
		ch.h_ctrl.p = h + sl.h_ctrl;
	}
	// Each chunk's data, sigma and region canvases: cleared on the device,
	// then every galaxy's rows packed into a pinned staging buffer, copied
	// up with one transfer per staging buffer and placed in their canvas
	// slots by k_cat_scatter (the canvas beyond a galaxy keeps region 0, so
	// its sigma there is never read); PSFs and their reversals packed per
	// chunk.  Chunks are independent: host threads take them in turn, each
	// with its own stream and two staging buffers, so packing one overlaps
	// the transfer of the other.
	{
		const int dev = c->engine->device;
		size_t maxw = 1;
		for (const CatGalaxy &G : c->gal) maxw = std::max<size_t>(maxw, G.w);
		constexpr int MAX_PIECES = 4096;
		const size_t head = MAX_PIECES * sizeof(CatPiece);
		const size_t stage = std::max<size_t>((size_t)8 << 20, head + maxw * 16);
		const size_t cap = (stage - head) / 8;  // doubles per staging buffer
		std::atomic<size_t> next{0};
		std::atomic<int> status{PF_OK};
		std::mutex err_mu;
		std::string err_msg;
		auto worker = [&]() {
			cudaError_t e = cudaSetDevice(dev);
			cudaStream_t st = nullptr;
			cudaEvent_t done[2] = {};
			if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
			for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
			HostBuf hb;
			DevBuf db;
			if (e == cudaSuccess) e = ensure(hb, 2 * stage);
			if (e == cudaSuccess) e = ensure(db, 2 * stage);
			int half = 0, np = 0, maxpix = 0;
			bool used[2] = {false, false};
			size_t nv = 0;
			auto pieces = [&]() { return reinterpret_cast<CatPiece *>(hb.as<char>() + half * stage); };
			auto values = [&]() { return reinterpret_cast<double *>(hb.as<char>() + half * stage + head); };
			auto flush = [&](CatChunk &ch) {
				if (np == 0 || e != cudaSuccess) return;
				char *hs = hb.as<char>() + half * stage, *ds = db.as<char>() + half * stage;
				e = cudaMemcpyAsync(ds, hs, head + nv * 8, cudaMemcpyHostToDevice, st);
				if (e == cudaSuccess)
					e = launch_cat_scatter(reinterpret_cast<const CatPiece *>(ds), np, maxpix,
					                       reinterpret_cast<const double *>(ds + head), ch.data.as<double>(),
					                       ch.sigma.as<double>(), ch.region.as<uint8_t>(), st);
				if (e == cudaSuccess) e = cudaEventRecord(done[half], st);
				used[half] = true;
				half ^= 1;
				if (e == cudaSuccess && used[half]) e = cudaEventSynchronize(done[half]);
				np = 0;
				nv = 0;
				maxpix = 0;
			};
			for (size_t k = next++; k < c->chunks.size() && status == PF_OK && e == cudaSuccess; k = next++) {
				CatChunk &ch = *c->chunks[k];
				const int C = (int)ch.members.size();
				const size_t nout = ch.nout(), nk = (size_t)ch.pw * ch.ph;
				e = cudaMemsetAsync(ch.data.p, 0, nout * C * 8, st);
				if (e == cudaSuccess) e = cudaMemsetAsync(ch.sigma.p, 0, nout * C * 8, st);
				if (e == cudaSuccess) e = cudaMemsetAsync(ch.region.p, 0, nout * C, st);
				for (int i = 0; i < C && e == cudaSuccess; i++) {
					const CatGalaxy &G = c->gal[ch.members[i]];
					// rows of this galaxy that fit one staging buffer (at least one: the
					// buffer holds the widest row)
					const unsigned rp = (unsigned)std::min<size_t>(G.h, cap / 2 / G.w);
					for (unsigned r0 = 0; r0 < G.h && e == cudaSuccess; r0 += rp) {
						const unsigned rows = std::min(rp, G.h - r0);
						const size_t n = (size_t)G.w * rows;
						if (np == MAX_PIECES || nv + 2 * n > cap) flush(ch);
						if (e != cudaSuccess) break;
						CatPiece &pc = pieces()[np++];
						pc.dst = (unsigned long long)i * nout + (unsigned long long)r0 * ch.W;
						pc.src = nv;
						pc.w = (int)G.w;
						pc.rows = (int)rows;
						pc.W = (int)ch.W;
						pc.pad_ = 0;
						std::memcpy(values() + nv, G.data.data() + (size_t)r0 * G.w, n * 8);
						std::memcpy(values() + nv + n, G.sigma.data() + (size_t)r0 * G.w, n * 8);
						nv += 2 * n;
						maxpix = std::max(maxpix, (int)std::min<size_t>(n, 1u << 30));
					}
				}
				flush(ch);
				// the chunk's PSFs and their reversals (FP32), through staging buffers
				// too, as many galaxies per copy as fit
				const size_t per_copy = std::max<size_t>(1, stage / (2 * nk * 4));
				for (size_t g0 = 0; g0 < (size_t)C && e == cudaSuccess; g0 += per_copy) {
					const size_t ng = std::min(per_copy, (size_t)C - g0);
					if (2 * ng * nk * 4 > stage) {  // one PSF larger than a staging buffer
						e = cudaErrorInvalidValue;
						break;
					}
					float *hs = reinterpret_cast<float *>(hb.as<char>() + half * stage), *hr = hs + ng * nk;
					for (size_t i = 0; i < ng; i++) {
						const CatGalaxy &G = c->gal[ch.members[g0 + i]];
						for (size_t q = 0; q < nk; q++) {
							hs[i * nk + q] = (float)G.psf[q];
							hr[i * nk + q] = (float)G.psf[nk - 1 - q];
						}
					}
					e = cudaMemcpyAsync(ch.psf32.as<float>() + g0 * nk, hs, ng * nk * 4, cudaMemcpyHostToDevice, st);
					if (e == cudaSuccess)
						e = cudaMemcpyAsync(ch.psfrev32.as<float>() + g0 * nk, hr, ng * nk * 4, cudaMemcpyHostToDevice, st);
					if (e == cudaSuccess) e = cudaEventRecord(done[half], st);
					used[half] = true;
					half ^= 1;
					if (e == cudaSuccess && used[half]) e = cudaEventSynchronize(done[half]);
				}
			}
			// the staging buffers are freed below: wait for their transfers
			if (st) {
				cudaError_t e2 = cudaStreamSynchronize(st);
				if (e == cudaSuccess) e = e2;
			}
			for (cudaEvent_t ev : done)
				if (ev) cudaEventDestroy(ev);
			if (st) cudaStreamDestroy(st);
			if (e != cudaSuccess) {
				std::lock_guard<std::mutex> g(err_mu);
				err_msg = cudaGetErrorString(e);
				status = PF_E_CUDA;
			}
		};
		const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
		const size_t nthreads = std::max<size_t>(1, std::min<size_t>(std::min<size_t>(hw, 8), c->chunks.size()));
		std::vector<std::thread> pool;
		for (size_t t = 1; t < nthreads; t++) pool.emplace_back(worker);
		worker();
		for (auto &t : pool) t.join();
		if (status != PF_OK) return set_error(PF_E_CUDA, "catalogue inputs: " + err_msg);
	}
	if (cat_log_on()) fprintf(stderr, "[profit_b200 catalogue] inputs uploaded: %.3f s\n", cat_now() - t_build);
	c->nprof = (int)params.size();
	PF_CUDA(ensure(c->params, params.size() * sizeof(ProfileParams)));
	PF_CUDA(cudaMemcpy(c->params.p, params.data(), params.size() * sizeof(ProfileParams), cudaMemcpyHostToDevice));
	PF_CUDA(ensure(c->pad, pad.size() * sizeof(int2)));
	PF_CUDA(cudaMemcpy(c->pad.p, pad.data(), pad.size() * sizeof(int2), cudaMemcpyHostToDevice));
	PF_CUDA(ensure(c->dev, params.size() * sizeof(DevProfile)));
	PF_CUDA(ensure(c->fprof, params.size() * sizeof(FProfile)));
	PF_CUDA(ensure(c->lum, params.size() * LUM_SLOTS * sizeof(double)));

	// lanes: engines of their own (stream, scratch, queue); chunks assigned
	// greedily by drawing pixels to the least loaded lane
	if (c->lanes.empty()) c->lanes.push_back(c->engine);
	while ((int)c->lanes.size() < CAT_LANES) {
		pf_model *e = nullptr;
		PF_TRY(pf_model_create(1, 1, &e));
		e->precision = PF_FP32;
		c->lanes.push_back(e);
	}
	if (!c->fork) PF_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
	while ((int)c->joins.size() < CAT_LANES) {
		cudaEvent_t e;
		PF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		c->joins.push_back(e);
	}
	{
		std::vector<double> load(CAT_LANES, 0.0);
		for (auto &chp : c->chunks) {
			int best = 0;
			for (int l = 1; l < CAT_LANES; l++)
				if (load[l] < load[best]) best = l;
			chp->lane = best;
			load[best] += (double)chp->npix() * chp->members.size() * chp->levels;
		}
	}
	// each lane's scratch and queue for its largest chunk, so nothing is
	// reallocated while chunks are queued; lane 0 also runs every chunk on
	// its own (the eager first call, re-runs after an overflow)
	c->lane_qpix.assign(CAT_LANES, 0);
	c->max_levels = 1;
	for (int lane = 0; lane < CAT_LANES; lane++) {
		pf_model *m = c->lanes[lane];
		size_t conv = 0, model = 0, seed = 0, jac = 0, parts = 0, qpix = 0, jp = 0;
		int levels = 1, maxprof = 0, maxc = 1;
		for (auto &chp : c->chunks) {
			const CatChunk &ch = *chp;
			if (lane != 0 && ch.lane != lane) continue;
			const size_t C = ch.members.size();
			maxc = std::max(maxc, (int)C);
			conv = std::max(conv, ch.npix() * 4 * C);
			model = std::max(model, ch.nout() * 8 * C);
			seed = std::max(seed, ch.nout() * 4 * C);
			jac = std::max(jac, ch.npix() * (size_t)ch.nt * ch.nprof * sizeof(double));
			parts = std::max(parts, C * NPARTS * sizeof(double2));
			qpix = std::max(qpix, ch.npix() * C);
			jp = std::max(jp, (size_t)ch.nprof *
			                            jac_reduce_blocks(ch.W + 2 * (ch.pw / 2), ch.H + 2 * (ch.ph / 2), ch.nprof) * NTAN * 8);
			levels = std::max(levels, ch.levels);
			maxprof = std::max(maxprof, ch.nprof);
		}
		PF_CUDA(ensure(m->d_conv32, conv));
		PF_CUDA(ensure(m->d_plain32, conv));
		PF_CUDA(ensure(m->d_gconv, conv));
		PF_CUDA(ensure(m->d_gplain, conv));
		PF_CUDA(ensure(m->d_model64, model));
		PF_CUDA(ensure(m->d_wseed, seed));
		PF_CUDA(ensure(m->d_jac, jac));
		PF_CUDA(ensure(m->d_partials, parts));
		PF_CUDA(ensure(m->d_convsplit, (size_t)64 << 20));
		PF_CUDA(ensure(m->d_jac_partials, jp));
		void *before = m->d_jac_tickets.p;
		PF_CUDA(ensure(m->d_jac_tickets, (size_t)maxprof * sizeof(unsigned)));
		if (m->d_jac_tickets.p != before)
			PF_CUDA(cudaMemsetAsync(m->d_jac_tickets.p, 0, m->d_jac_tickets.bytes, m->stream));
		unsigned *like_tk;
		PF_TRY(like_tickets(m, maxc, &like_tk));
		Analysis a;
		a.levels = levels;
		QueueSet q;
		PF_TRY(prepare_queue(m, a, qpix, q, nullptr, nullptr, false, true, true));  // sizes the kind-group buffer too
		PF_CUDA(cudaStreamSynchronize(m->stream));
		c->lane_qpix[lane] = qpix;
		c->max_levels = std::max(c->max_levels, levels);
	}
	const double t_conv = cat_now();
	if (cat_log_on()) fprintf(stderr, "[profit_b200 catalogue] lanes and scratch: %.3f s\n", t_conv - t_build);
	PF_TRY(cat_pick_convolvers(c));
	if (cat_log_on()) {
		int nfft = 0;
		for (auto &ch : c->chunks) nfft += ch->fft ? 1 : 0;
		fprintf(stderr, "[profit_b200 catalogue] convolver per batch: %.3f s (%d of %zu batches through FFTs)\n",
		        cat_now() - t_conv, nfft, c->chunks.size());
	}
	c->built = true;
	return PF_OK;
}

// Gives every lane the largest queue capacities any lane has grown to, and
// sizes their queues for them, so that a recorded call finds them all at
// what the eager run (on lane 0) needed.
int cat_share_capacities(pf_catalogue *c)
{
	std::vector<uint32_t> mx(MAX_LEVELS, 0);
	for (pf_model *m : c->lanes)
		for (int l = 0; l < MAX_LEVELS && l < (int)m->caps.size(); l++) mx[l] = std::max(mx[l], m->caps[l]);
	for (int lane = 0; lane < (int)c->lanes.size(); lane++) {
		pf_model *m = c->lanes[lane];
		m->caps = mx;
		Analysis a;
		a.levels = c->max_levels;
		QueueSet q;
		PF_TRY(prepare_queue(m, a, c->lane_qpix[lane], q, nullptr, nullptr, false, false, true));
	}
	return PF_OK;
}

// Every lane's capacities, in lane order (what a recorded call depends on).
std::vector<uint32_t> cat_capacities(const pf_catalogue *c)
{
	std::vector<uint32_t> v;
	for (const pf_model *m : c->lanes) v.insert(v.end(), m->caps.begin(), m->caps.end());
	return v;
}

// Queues one chunk's pipeline (prologue already run); results and queue
// counters land in the chunk's pinned buffers when the stream gets there.
int cat_enqueue_chunk(pf_catalogue *c, CatChunk &ch, int lane)
{
	pf_model *m = c->lanes[lane];
	cudaStream_t s = m->stream;
	const int C = (int)ch.members.size();
	const Analysis a = cat_analysis(ch);
	const size_t npix = ch.npix(), nout = ch.nout();
	QueueSet q;
	PF_TRY(prepare_queue(m, a, npix * C, q, nullptr, nullptr, false, true, ch.ak));
	// FP64 tangent planes: catalogue galaxies are often a few pixels across
	// and bright, so most of their flux sits in subsampled pixels whose cells
	// cancel in the position and shape tangents
	float *conv = m->d_conv32.as<float>(), *plain = m->d_plain32.as<float>();
	double *jac = m->d_jac.as<double>();
	float *gconv = m->d_gconv.as<float>(), *gplain = m->d_gplain.as<float>(), *wseed = m->d_wseed.as<float>();
	double *model64 = m->d_model64.as<double>();
	const FProfile *fprof = c->fprof.as<FProfile>() + ch.p0;
	const DevProfile *dev = c->dev.as<DevProfile>() + ch.p0;
	PF_CUDA(launch_pixels32(fprof, ch.prof_begin.as<int>(), C, a.dw, a.dh, 1.0, 1.0, conv, plain, jac, ch.nt, ch.ak, q,
	                        s, nullptr, ch.extent.as<int2>()));
	PF_CUDA(launch_levels32(fprof, a.levels, (unsigned)npix, conv, plain, jac, ch.nt, ch.ak, ch.cusps, q, s));
	PF_TRY(cat_conv_forward(m, ch, a, ch.fft, conv, plain, model64, s));
	PF_CUDA(launch_loglike64_batch(model64, ch.data.as<double>(), ch.sigma.as<double>(), ch.region.as<uint8_t>(),
	                               (int)nout, C, (int)nout, m->d_partials.as<double2>(), like_parts((int)nout, C),
	                               ch.ll.as<double>(), wseed, s, m->d_like_tickets.as<unsigned>()));
	if (ch.plain) PF_CUDA(launch_embed_seed(wseed, a.ow, a.oh, a.padx, a.pady, a.dw, a.dh, C, gplain, s));
	PF_TRY(cat_conv_adjoint(m, ch, a, ch.fft, wseed, gconv, s));
	PF_CUDA(launch_jac_reduce(jac, gconv, gplain, fprof, ch.prof_batch.as<int>(), ch.nprof, a.dw, a.dh, 1.0, 1.0,
	                          ch.nt, m->d_jac_partials.as<double>(), m->d_jac_tickets.as<unsigned>(),
	                          ch.T.as<double>(), s, nullptr, ch.extent.as<int2>()));
	PF_CUDA(launch_cat_gradient(dev, ch.nprof, ch.T.as<double>(), ch.grad_off.as<int>(), ch.grad.as<double>(), s));
	PF_CUDA(cudaMemcpyAsync(ch.h_ll.p, ch.ll.p, (size_t)C * 8, cudaMemcpyDeviceToHost, s));
	PF_CUDA(cudaMemcpyAsync(ch.h_grad.p, ch.grad.p, (size_t)std::max(ch.ngrad, 1) * 8, cudaMemcpyDeviceToHost, s));
	PF_CUDA(cudaMemcpyAsync(ch.h_ctrl.p, m->d_ctrl.p, CTRL_WORDS * 4, cudaMemcpyDeviceToHost, s));
	return PF_OK;
}

}  // namespace

extern "C" {

int pf_catalogue_create(pf_catalogue **out)
{
	if (!out) return set_error(PF_E_INVALID, "null output pointer");
	pf_catalogue *c = new pf_catalogue();
	int st = pf_model_create(1, 1, &c->engine);
	if (st != PF_OK) {
		delete c;
		return st;
	}
	c->engine->precision = PF_FP32;
	for (auto &e : c->ev) cudaEventCreate(&e);
	*out = c;
	return PF_OK;
}

int pf_catalogue_destroy(pf_catalogue *c)
{
	if (!c) return PF_OK;
	if (c->graph) cudaGraphExecDestroy(c->graph);
	c->chunks.clear();
	for (auto &e : c->ev)
		if (e) cudaEventDestroy(e);
	if (c->fork) cudaEventDestroy(c->fork);
	for (cudaEvent_t e : c->joins) cudaEventDestroy(e);
	for (size_t l = 1; l < c->lanes.size(); l++) pf_model_destroy(c->lanes[l]);
	pf_model_destroy(c->engine);
	delete c;
	return PF_OK;
}

int pf_catalogue_set_magzero(pf_catalogue *c, double magzero)
{
	if (!c) return set_error(PF_E_INVALID, "null catalogue");
	c->magzero = magzero;
	return PF_OK;
}

int pf_catalogue_set_convolver(pf_catalogue *c, const char *name)
{
	if (!c || !name) return set_error(PF_E_INVALID, "null argument");
	int mode;
	if (!std::strcmp(name, "auto")) mode = CAT_CONV_AUTO;
	else if (!std::strcmp(name, "brute")) mode = CAT_CONV_BRUTE;
	else if (!std::strcmp(name, "fft")) mode = CAT_CONV_FFT;
	else return set_error(PF_E_INVALID, std::string("unknown catalogue convolver: ") + name);
	if (mode != c->conv_mode) {
		c->conv_mode = mode;
		c->built = false;  // chunks pick again at the next evaluation
	}
	return PF_OK;
}

int pf_catalogue_convolvers(const pf_catalogue *c, int *fft_chunks, int *chunks)
{
	if (!c || !fft_chunks || !chunks) return set_error(PF_E_INVALID, "null argument");
	*chunks = (int)c->chunks.size();
	*fft_chunks = 0;
	for (const auto &ch : c->chunks) *fft_chunks += ch->fft ? 1 : 0;
	return PF_OK;
}

int pf_catalogue_add_galaxy(pf_catalogue *c, unsigned width, unsigned height, const double *data,
                            const double *sigma, const double *psf, unsigned psf_w, unsigned psf_h, int *index)
{
	if (!c || !data || !sigma || !psf) return set_error(PF_E_INVALID, "null argument");
	if (width == 0 || height == 0 || psf_w == 0 || psf_h == 0) return set_error(PF_E_INVALID, "empty image or psf");
	if (width > 4096 || height > 4096 || psf_w > 255 || psf_h > 255)
		return set_error(PF_E_INVALID, "catalogue galaxies are limited to 4096 x 4096 images and 255 x 255 PSFs");
	CatGalaxy G;
	G.w = width;
	G.h = height;
	G.pw = psf_w;
	G.ph = psf_h;
	G.data.assign(data, data + (size_t)width * height);
	G.sigma.assign(sigma, sigma + (size_t)width * height);
	for (double s : G.sigma)
		if (!(s > 0)) return set_error(PF_E_INVALID, "sigma must be positive");
	double sum = 0;
	for (size_t k = 0; k < (size_t)psf_w * psf_h; k++) sum += psf[k];
	if (!(sum > 0)) return set_error(PF_E_INVALID, "psf must have a positive sum");
	G.psf.assign(psf, psf + (size_t)psf_w * psf_h);
	for (double &v : G.psf) v /= sum;
	c->gal.push_back(std::move(G));
	c->built = false;
	if (index) *index = (int)c->gal.size() - 1;
	return PF_OK;
}

int pf_catalogue_add_profile(pf_catalogue *c, int galaxy, const char *kind, int n_params, const char *const *names,
                             const double *values)
{
	if (!c || !kind || (n_params > 0 && (!names || !values))) return set_error(PF_E_INVALID, "null argument");
	if (galaxy < 0 || galaxy >= (int)c->gal.size()) return set_error(PF_E_INVALID, "galaxy index out of range");
	int k = kind_from_name(kind);
	if (k < 0) return set_error(PF_E_INVALID, std::string("Unknown profile name: ") + kind);
	if (!is_radial_kind(k)) return set_error(PF_E_INVALID, "catalogue galaxies take radial profiles only");
	ProfileParams p = default_params(k);
	p.convolve = 1;
	for (int i = 0; i < n_params; i++) PF_TRY(cat_set_param(p, names[i], values[i]));
	const char *err = validate_profile(p, true);
	if (err) return set_error(PF_E_INVALID, err);
	if (!params_valid(p)) return set_error(PF_E_INVALID, "invalid profile parameters");
	if (p.kind == PK_SERSIC && p.rescale_flux) return set_error(PF_E_INVALID, "gradients with rescale_flux are not available");
	if (!p.adjust && !p.rough && (p.resolution == 0 || p.resolution > 16))
		return set_error(PF_E_INVALID, "resolution must be in [1, 16] when adjust is false");
	if (p.max_recursions + 1 > (unsigned)MAX_LEVELS) return set_error(PF_E_INVALID, "max_recursions above 15 is not supported");
	c->gal[galaxy].profiles.push_back(p);
	c->built = false;
	return PF_OK;
}

int pf_catalogue_set_values(pf_catalogue *c, const double *values)
{
	if (!c || !values) return set_error(PF_E_INVALID, "null argument");
	// every profile checked before any is changed
	size_t at = 0;
	for (size_t g = 0; g < c->gal.size(); g++)
		for (const ProfileParams &p0 : c->gal[g].profiles) {
			ProfileParams p = p0;
			const int n = 6 + shape_count(p.kind);
			for (int k = 0; k < n; k++) *cat_value_slot(p, k) = values[at + k];
			at += n;
			const char *err = validate_profile(p, true);
			if (err || !params_valid(p))
				return set_error(PF_E_INVALID, "galaxy " + std::to_string(g) + ": " +
				                                   (err ? err : "invalid profile parameters"));
		}
	at = 0;
	for (auto &G : c->gal)
		for (ProfileParams &p : G.profiles) {
			const int n = 6 + shape_count(p.kind);
			for (int k = 0; k < n; k++) *cat_value_slot(p, k) = values[at + k];
			at += n;
		}
	c->params_dirty = c->built;
	return PF_OK;
}

int pf_catalogue_get_values(pf_catalogue *c, double *values)
{
	if (!c || !values) return set_error(PF_E_INVALID, "null argument");
	size_t at = 0;
	for (auto &G : c->gal)
		for (ProfileParams &p : G.profiles) {
			const int n = 6 + shape_count(p.kind);
			for (int k = 0; k < n; k++) values[at + k] = *cat_value_slot(p, k);
			at += n;
		}
	return PF_OK;
}

int pf_catalogue_size(pf_catalogue *c, int *n_galaxies, int *n_grad)
{
	if (!c) return set_error(PF_E_INVALID, "null catalogue");
	int total = 0;
	for (auto &G : c->gal)
		for (auto &p : G.profiles) total += 6 + shape_count(p.kind);
	if (n_galaxies) *n_galaxies = (int)c->gal.size();
	if (n_grad) *n_grad = total;
	return PF_OK;
}

int pf_catalogue_gradient_offset(pf_catalogue *c, int galaxy, int *offset, int *count)
{
	if (!c) return set_error(PF_E_INVALID, "null catalogue");
	if (galaxy < 0 || galaxy >= (int)c->gal.size()) return set_error(PF_E_INVALID, "galaxy index out of range");
	int off = 0;
	for (int g = 0; g < galaxy; g++)
		for (auto &p : c->gal[g].profiles) off += 6 + shape_count(p.kind);
	int n = 0;
	for (auto &p : c->gal[galaxy].profiles) n += 6 + shape_count(p.kind);
	if (offset) *offset = off;
	if (count) *count = n;
	return PF_OK;
}

int pf_catalogue_loglike_grad(pf_catalogue *c, double *loglike, double *grad)
{
	if (!c || !loglike) return set_error(PF_E_INVALID, "null argument");
	if (c->gal.empty()) return PF_OK;
	for (auto &G : c->gal)
		if (G.profiles.empty()) return set_error(PF_E_STATE, "a catalogue galaxy has no profiles");
	PF_TRY(ensure_stream(c->engine));
	const double t_call = cat_now();
	if (!c->built) {
		PF_TRY(cat_build(c));
		if (cat_log_on())
			fprintf(stderr, "[profit_b200 catalogue] build: %.3f s (%zu batches)\n", cat_now() - t_call, c->chunks.size());
	}
	pf_model *m = c->engine;
	if (c->params_dirty) {
		// new values (pf_catalogue_set_values): the profile records in chunk
		// order again; the recorded call reads them from the same buffer
		std::vector<ProfileParams> params;
		params.reserve(c->nprof);
		for (auto &chp : c->chunks) {
			chp->cusps = 0;
			for (int gi : chp->members)
				for (const ProfileParams &p : c->gal[gi].profiles) {
					params.push_back(p);
					if (p.kind == PK_SERSIC && p.adjust && p.nser > 1) chp->cusps++;
				}
		}
		PF_CUDA(cudaMemcpy(c->params.p, params.data(), params.size() * sizeof(ProfileParams), cudaMemcpyHostToDevice));
		c->params_dirty = false;
	}
	cudaStream_t s = m->stream;
	PF_CUDA(cudaEventRecord(c->ev[0], s));
	ModelGeom g;
	g.magzero = c->magzero;
	g.sx = g.sy = g.img_sx = g.img_sy = 1;
	g.offx = g.offy = 0;
	g.finesampling = 1;
	// The prologue, then every chunk: on lane 0 alone (the eager call, whose
	// convolution tuning then times each candidate on an otherwise idle GPU),
	// or on the chunks' own lanes, forked from and joined back into lane 0's
	// stream (the recorded call).
	auto enqueue_chunks = [&](const std::vector<CatChunk *> &list, bool on_lanes) -> int {
		if (on_lanes) {
			PF_CUDA(cudaEventRecord(c->fork, s));
			for (int l = 1; l < (int)c->lanes.size(); l++) PF_CUDA(cudaStreamWaitEvent(c->lanes[l]->stream, c->fork, 0));
		}
		for (CatChunk *ch : list) PF_TRY(cat_enqueue_chunk(c, *ch, on_lanes ? ch->lane : 0));
		if (on_lanes)
			for (int l = 1; l < (int)c->lanes.size(); l++) {
				PF_CUDA(cudaEventRecord(c->joins[l], c->lanes[l]->stream));
				PF_CUDA(cudaStreamWaitEvent(s, c->joins[l], 0));
			}
		return PF_OK;
	};
	std::vector<CatChunk *> all;
	for (auto &chp : c->chunks) all.push_back(chp.get());
	auto enqueue_all = [&](bool on_lanes) -> int {
		PF_CUDA(launch_cat_prologue(c->params.as<ProfileParams>(), c->pad.as<int2>(), c->nprof, g,
		                            c->lum.as<double>(), c->dev.as<DevProfile>(), c->fprof.as<FProfile>(), s));
		return enqueue_chunks(all, on_lanes);
	};
	std::vector<CatChunk *> todo = all;
	const bool replay = c->graph && c->graph_caps == cat_capacities(c);
	bool retried = false;
	for (int attempt = 0; attempt < 8 && !todo.empty(); attempt++) {
		const bool on_lanes = attempt == 0 && replay;
		// every chunk is judged against the capacities of the lane it ran on,
		// as they were when it ran (one chunk's growth must not hide another's
		// overflow)
		std::vector<std::vector<uint32_t>> used;
		for (pf_model *e : c->lanes) used.push_back(e->caps);
		if (on_lanes) {
			PF_CUDA(cudaGraphLaunch(c->graph, s));
			note_launches((int)c->graph_kernels);
		}
		else if (attempt == 0) {
			PF_TRY(enqueue_all(false));
		}
		else {
			PF_TRY(enqueue_chunks(todo, false));
		}
		PF_CUDA(cudaStreamSynchronize(s));
		std::vector<CatChunk *> again;
		for (CatChunk *ch : todo) {
			const uint32_t *ctrl = ch->h_ctrl.as<uint32_t>();
			if (ctrl[MAX_LEVELS] & 2u) return set_error(PF_E_CAPACITY, "recursion deeper than the configured levels");
			const int lane = on_lanes ? ch->lane : 0;
			bool over = false;
			for (int l = 0; l < ch->levels; l++)
				if (ctrl[l] > used[lane][l]) {
					over = true;
					uint64_t want = (uint64_t)ctrl[l] + ctrl[l] / 2 + 1024;
					if (want > (1ull << 30)) return set_error(PF_E_CAPACITY, "subsampling work queue overflow");
					// the re-run goes to lane 0
					c->lanes[0]->caps[l] = std::max(c->lanes[0]->caps[l], (uint32_t)want);
				}
			if (over) again.push_back(ch);
		}
		if (!again.empty()) retried = true;
		todo.swap(again);
	}
	if (!todo.empty()) return set_error(PF_E_CAPACITY, "subsampling work queue kept overflowing");
	if (retried && c->graph) {
		cudaGraphExecDestroy(c->graph);  // captured with capacities that no longer hold
		c->graph = nullptr;
	}
	if (cat_log_on() && !replay)
		fprintf(stderr, "[profit_b200 catalogue] evaluation without the recorded call: %.3f s since the call began\n",
		        cat_now() - t_call);
	if (!replay && !retried && m->use_graphs) {
		// record the call that just ran (every choice it made is cached now)
		// for the next calls, with the chunks on their lanes; nothing runs
		// during the capture
		if (c->graph) cudaGraphExecDestroy(c->graph);
		c->graph = nullptr;
		PF_TRY(cat_share_capacities(c));
		for (pf_model *e : c->lanes) PF_CUDA(cudaStreamSynchronize(e->stream));
		const unsigned long long before = g_launches.load();
		cudaGraph_t graph = nullptr;
		PF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
		const int st = enqueue_all(true);
		const cudaError_t ce = cudaStreamEndCapture(s, &graph);
		c->graph_kernels = g_launches.load() - before;
		g_launches -= c->graph_kernels;
		if (st == PF_OK && ce == cudaSuccess && graph && cudaGraphInstantiate(&c->graph, graph, 0) == cudaSuccess)
			c->graph_caps = cat_capacities(c);
		else
			c->graph = nullptr;
		if (graph) cudaGraphDestroy(graph);
		cudaGetLastError();
	}
	PF_CUDA(cudaEventRecord(c->ev[1], s));
	PF_CUDA(cudaEventSynchronize(c->ev[1]));
	if (cat_log_on() && !replay)
		fprintf(stderr, "[profit_b200 catalogue] call with recording: %.3f s\n", cat_now() - t_call);
	for (auto &chp : c->chunks) {
		const CatChunk &ch = *chp;
		const double *hl = ch.h_ll.as<double>(), *hg = ch.h_grad.as<double>();
		for (size_t i = 0; i < ch.members.size(); i++) {
			const int gi = ch.members[i];
			loglike[gi] = hl[i];
			if (grad) {
				int n = 0;
				for (auto &p : c->gal[gi].profiles) n += 6 + shape_count(p.kind);
				std::memcpy(grad + c->grad_off[gi], hg + ch.member_grad_off[i], (size_t)n * 8);
			}
		}
	}
	cudaEventElapsedTime(&c->last_ms, c->ev[0], c->ev[1]);
	cudaGetLastError();
	return PF_OK;
}

int pf_catalogue_last_time(pf_catalogue *c, float *ms)
{
	if (!c || !ms) return set_error(PF_E_INVALID, "null argument");
	*ms = c->last_ms;
	return PF_OK;
}

}  // extern "C"
