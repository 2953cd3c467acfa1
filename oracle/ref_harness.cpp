/*
 * ORACLE (test infrastructure only): a flat C interface over the reference's
 * own libprofit C++ (profit::Model, src/libprofit/src/profit/model.h:55-421),
 * compiled in place from the reference sources by oracle/Makefile.
 *
 * It plays the role that src/r_profit.cpp:549-680 (R_profit_make_model) plays
 * for R: build a Model, add profiles, set parameters by name, set the PSF and
 * convolver, evaluate.  Nothing here re-implements libprofit; it only forwards.
 * Errors (profit::exception and std::exception) become a -1 status plus a
 * thread-local message, as R_profit_make_model turns them into Rf_error.
 */
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "profit/profit.h"
#include "profit/radial.h"
#include "profit/convolve.h"

using namespace profit;

namespace {

thread_local std::string g_last_error;

struct RefModel {
	Model model;
	std::vector<ProfilePtr> profiles;
	RefModel(unsigned w, unsigned h) : model(w, h) {}
};

template <typename F>
int guarded(F &&f)
{
	try {
		f();
		return 0;
	} catch (const std::exception &e) {
		g_last_error = e.what();
		return -1;
	}
}

} // namespace

extern "C" {

const char *pfref_last_error(void) { return g_last_error.c_str(); }

void *pfref_model_new(unsigned width, unsigned height)
{
	return new RefModel(width, height);
}

void pfref_model_free(void *m) { delete static_cast<RefModel *>(m); }

int pfref_add_profile(void *m, const char *name)
{
	auto *rm = static_cast<RefModel *>(m);
	int idx = -1;
	int st = guarded([&] {
		rm->profiles.push_back(rm->model.add_profile(name));
		idx = static_cast<int>(rm->profiles.size()) - 1;
	});
	return st == 0 ? idx : -1;
}

/* "name = value", parsed by Profile::parameter(const std::string &) */
int pfref_profile_set(void *m, int idx, const char *spec)
{
	auto *rm = static_cast<RefModel *>(m);
	if (idx < 0 || idx >= (int)rm->profiles.size()) {
		g_last_error = "profile index out of range";
		return -1;
	}
	return guarded([&] { rm->profiles[idx]->parameter(std::string(spec)); });
}

int pfref_profile_set_double(void *m, int idx, const char *name, double v)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] { rm->profiles.at(idx)->parameter(std::string(name), v); });
}

int pfref_profile_set_uint(void *m, int idx, const char *name, unsigned v)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] { rm->profiles.at(idx)->parameter(std::string(name), v); });
}

int pfref_profile_set_bool(void *m, int idx, const char *name, int v)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] { rm->profiles.at(idx)->parameter(std::string(name), (bool)v); });
}

int pfref_set_psf(void *m, const double *psf, unsigned w, unsigned h)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] {
		std::vector<double> data(psf, psf + (size_t)w * h);
		rm->model.set_psf(Image(std::move(data), w, h));
	});
}

void pfref_set_magzero(void *m, double mz) { static_cast<RefModel *>(m)->model.set_magzero(mz); }

void pfref_set_scale(void *m, double sx, double sy)
{
	auto *rm = static_cast<RefModel *>(m);
	rm->model.set_image_pixel_scale({sx, sy});
}

void pfref_set_psf_scale(void *m, double sx, double sy)
{
	auto *rm = static_cast<RefModel *>(m);
	rm->model.set_psf_pixel_scale({sx, sy});
}

int pfref_set_finesampling(void *m, unsigned fs)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] { rm->model.set_finesampling(fs); });
}

void pfref_set_return_finesampled(void *m, int v) { static_cast<RefModel *>(m)->model.set_return_finesampled(v != 0); }
void pfref_set_crop(void *m, int v) { static_cast<RefModel *>(m)->model.set_crop(v != 0); }
void pfref_set_omp_threads(void *m, unsigned t) { static_cast<RefModel *>(m)->model.set_omp_threads(t); }
void pfref_set_adjust_mask(void *m, int v) { static_cast<RefModel *>(m)->model.set_adjust_mask(v != 0); }

int pfref_set_mask(void *m, const unsigned char *mask, unsigned w, unsigned h)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] {
		std::vector<bool> data((size_t)w * h);
		for (size_t i = 0; i < data.size(); i++) data[i] = mask[i] != 0;
		rm->model.set_mask(Mask(std::move(data), w, h));
	});
}

/* type: "brute", "brute-old", "null" (FFTW is not available in this build) */
int pfref_set_convolver(void *m, const char *type, unsigned omp_threads)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] {
		ConvolverCreationPreferences prefs;
		prefs.omp_threads = omp_threads;
		rm->model.set_convolver(create_convolver(std::string(type), prefs));
	});
}

int pfref_drawing_dims(void *m, unsigned *w, unsigned *h)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] {
		auto d = rm->model.get_drawing_dimensions();
		*w = d.x;
		*h = d.y;
	});
}

/*
 * Evaluates the model.  `out` receives at most `cap` doubles, row-major with
 * x fastest (libprofit's Image layout); *w, *h get the image dimensions and
 * *ox, *oy the offset reported by Model::evaluate.
 */
int pfref_evaluate(void *m, double *out, size_t cap, unsigned *w, unsigned *h,
                   int *ox, int *oy)
{
	auto *rm = static_cast<RefModel *>(m);
	return guarded([&] {
		Point offset;
		Image img = rm->model.evaluate(offset);
		*w = img.getWidth();
		*h = img.getHeight();
		*ox = offset.x;
		*oy = offset.y;
		if (img.size() > cap) {
			throw std::runtime_error("output buffer too small");
		}
		std::memcpy(out, img.data(), sizeof(double) * img.size());
	});
}

/* Direct access to the shimmed special functions, as libprofit sees them. */
double pfref_qgamma(double p, double shape) { return profit::qgamma(p, shape); }
double pfref_pgamma(double q, double shape) { return profit::pgamma(q, shape); }
double pfref_gammafn(double x) { return profit::gammafn(x); }
double pfref_beta(double a, double b) { return profit::beta(a, b); }

struct pfref_integrand_ctx {
	double (*f)(double, void *);
	void *ud;
};

static double pfref_tramp(double x, void *ctx)
{
	auto *c = static_cast<pfref_integrand_ctx *>(ctx);
	return c->f(x, c->ud);
}

double pfref_integrate_qags(double (*f)(double, void *), void *ud, double a, double b)
{
	pfref_integrand_ctx c{f, ud};
	return profit::integrate_qags(pfref_tramp, a, b, &c);
}

double pfref_integrate_qagi(double (*f)(double, void *), void *ud, double a)
{
	pfref_integrand_ctx c{f, ud};
	return profit::integrate_qagi(pfref_tramp, a, &c);
}

#ifdef PROFIT_DEBUG
/*
 * Number of subsample_pixel calls per recursion level for profile `idx` during
 * the last evaluation (radial.cpp:70-78).  Returns the number of levels
 * written, or -1 if the profile is not radial.
 */
int pfref_integrations(void *m, int idx, int *counts, int max_levels)
{
	auto *rm = static_cast<RefModel *>(m);
	auto *rp = dynamic_cast<RadialProfile *>(rm->profiles.at(idx).get());
	if (!rp) return -1;
	auto ints = rp->get_integrations();
	int n = 0;
	for (int l = 0; l < max_levels; l++) counts[l] = 0;
	for (auto &kv : ints) {
		if (kv.first >= 0 && kv.first < max_levels) {
			counts[kv.first] = kv.second;
			if (kv.first + 1 > n) n = kv.first + 1;
		}
	}
	return n;
}
#endif

} // extern "C"
