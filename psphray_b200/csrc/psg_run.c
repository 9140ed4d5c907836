/* psg_run: a host driver in C over the library's C ABI (include/psg.h), with
 * the structure of one epoch of run_epoch() loop.c:87-160:
 *
 *   read the epoch's particles and sources (psystem_switch_epoch(),
 *   psystem.c:221, from a psphray-format file, reader-psphray.inc);
 *   set up units and tables (cfg_init(): units_init() units.c:66, ar_init()
 *   atomic-rate.c:66, xs_init() atomic-rate.c:93, the SPH kernel table);
 *   build the tree (rt_switch_epoch() raytrace.c:41);
 *   per tick: emit_rays(), trace(), deposit(), merge_pars(), update_pars()
 *   (loop.c:133-147), here psg_run_ticks_emit() over batches of ticks;
 *   write the output (psystem_write_output() psystem.c:598).
 *
 * The reference reads its switches and file names from a libconfig file;
 * this driver takes them on the command line:
 *
 *   psg_run SNAPSHOT RATES KERNEL NTICKS NRAY MYR OUTPUT [options]
 *     SNAPSHOT  psphray-format input (gas: pos, mass, sml, rho, ie, xHI, ye;
 *               type-5 particles: point sources, photons per unit time)
 *     RATES     atomic-rate table (atomic_rates_*.txt)
 *     KERNEL    kernel.akline
 *     NTICKS    ticks of the epoch; NRAY source rays per tick
 *     MYR       the epoch's duration in Myr (tick_time = MYR / NTICKS)
 *     OUTPUT    psphray-format output written at the end
 *   options: --batch K (ticks per library call, default 8), --energy EV
 *     (monochromatic photons, default 13.6), --blackbody T (instead: an
 *     8-line blackbody spectrum of temperature T over 1-10 Ry, log-spaced
 *     bins, photon-number weights), --isothermal, --hmf X (default 1:
 *     hydrogen only), --ppc P (default 8), --seed S, --device D, --resume
 *     (with --hmf below 1: take the helium fractions from the file's xHeI
 *     and xHeII blocks, as an earlier epoch's output wrote them, instead of
 *     deriving them from ye)
 *
 * Helium at load. The reference's live reader (psystem.c:330-360) reads
 * only ye and splits its electrons beyond x_HII into helium (HeII first,
 * then HeIII) and metals; psg_load_particles() does the same. Its resume
 * from an output (psystem.c:520-597) would read xHeI and xHeII back, but it
 * is compiled out (#if 0). --resume restores them: after the load, the
 * file's fractions replace the derived ones (psg_set_he_state). yeMET keeps
 * the load's value: an output's ye holds the hydrogen and helium electrons
 * only, so the split leaves the same (zero) metal electrons either way.
 *
 * Exit status: 0 done; 1 usage; 2 input files; 3 library or device error
 * (the library's message is printed). */
#define _POSIX_C_SOURCE 199309L
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include <string.h>
#include <time.h>

#include "psg.h"

static int usage(void) {
	fprintf(stderr,
			"usage: psg_run SNAPSHOT RATES KERNEL NTICKS NRAY MYR OUTPUT [--batch K] [--energy EV]\n"
			"               [--blackbody T] [--isothermal] [--hmf X] [--ppc P] [--seed S] [--device D]\n"
			"               [--resume]\n");
	return 1;
}

static int lib_fail(psg_context *ctx, int rc, const char *what) {
	fprintf(stderr, "psg_run: %s failed (%d): %s\n", what, rc, ctx ? psg_last_error(ctx) : "no context");
	return 3;
}

static double now_s(void) {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int main(int argc, char **argv) {
	if (argc < 8) return usage();
	const char *snap_path = argv[1], *rates_path = argv[2], *kernel_path = argv[3], *out_path = argv[7];
	const long long nticks = atoll(argv[4]), nray = atoll(argv[5]);
	const double myr = atof(argv[6]);
	long long batch = 8, ppc = 8, device = 0;
	unsigned long long seed = 20261203ull;
	double energy_ev = 13.6, hmf = 1.0, bb_T = 0.0;
	int isothermal = 0, resume = 0;
	for (int i = 8; i < argc; i++) {
		const char *a = argv[i];
		const int more = i + 1 < argc;
		if (!strcmp(a, "--isothermal")) isothermal = 1;
		else if (!strcmp(a, "--resume")) resume = 1;
		else if (!strcmp(a, "--batch") && more) batch = atoll(argv[++i]);
		else if (!strcmp(a, "--energy") && more) energy_ev = atof(argv[++i]);
		else if (!strcmp(a, "--blackbody") && more) bb_T = atof(argv[++i]);
		else if (!strcmp(a, "--hmf") && more) hmf = atof(argv[++i]);
		else if (!strcmp(a, "--ppc") && more) ppc = atoll(argv[++i]);
		else if (!strcmp(a, "--seed") && more) seed = strtoull(argv[++i], NULL, 10);
		else if (!strcmp(a, "--device") && more) device = atoll(argv[++i]);
		else return usage();
	}
	if (nticks <= 0 || nray <= 0 || !(myr > 0) || batch <= 0 || ppc <= 0 || !(hmf > 0 && hmf <= 1) ||
			!(energy_ev > 0) || bb_T < 0)
		return usage();

	/* the epoch's particles and sources */
	psg_snapshot snap;
	memset(&snap, 0, sizeof snap);
	if (psg_snapshot_read_header(snap_path, &snap) != PSG_OK || snap.ngas == 0) {
		fprintf(stderr, "psg_run: %s: not a psphray-format file with gas particles\n", snap_path);
		return 2;
	}
	const size_t n = snap.ngas, nsrc = snap.nsrc;
	if (nsrc == 0 || nsrc > PSG_MAX_SOURCES) {
		fprintf(stderr, "psg_run: %s: %zu sources (1 to %d supported)\n", snap_path, nsrc, PSG_MAX_SOURCES);
		return 2;
	}
	float *pos = malloc(sizeof(float) * 3 * n), *mass = malloc(sizeof(float) * n), *sml = malloc(sizeof(float) * n);
	float *rho = malloc(sizeof(float) * n), *ie = malloc(sizeof(float) * n), *xHI = malloc(sizeof(float) * n);
	float *ye = malloc(sizeof(float) * n), *src_pos = malloc(sizeof(float) * 3 * nsrc);
	int64_t *id = malloc(sizeof(int64_t) * n);
	double *ngammas = malloc(sizeof(double) * nsrc);
	if (!pos || !mass || !sml || !rho || !ie || !xHI || !ye || !src_pos || !id || !ngammas) {
		fprintf(stderr, "psg_run: out of host memory for %zu particles\n", n);
		return 2;
	}
	snap.pos = pos; snap.mass = mass; snap.sml = sml; snap.rho = rho; snap.ie = ie; snap.xHI = xHI;
	snap.ye = ye; snap.id = id; snap.src_pos = src_pos; snap.ngammas = ngammas;
	if (psg_snapshot_read(snap_path, &snap) != PSG_OK) {
		fprintf(stderr, "psg_run: %s: unreadable blocks\n", snap_path);
		return 2;
	}
	/* the helium fractions of an earlier epoch's output */
	double *lamHeI = NULL, *lamHeII = NULL;
	if (resume && hmf < 1.0) {
		psg_snapshot hs;
		memset(&hs, 0, sizeof hs);
		hs.ngas = snap.ngas;
		hs.nsrc = snap.nsrc;
		float *xHeI = malloc(sizeof(float) * n), *xHeII = malloc(sizeof(float) * n);
		lamHeI = malloc(sizeof(double) * n);
		lamHeII = malloc(sizeof(double) * n);
		if (!xHeI || !xHeII || !lamHeI || !lamHeII) {
			fprintf(stderr, "psg_run: out of host memory for %zu particles\n", n);
			return 2;
		}
		hs.xHeI = xHeI;
		hs.xHeII = xHeII;
		if (psg_snapshot_read(snap_path, &hs) != PSG_OK) {
			fprintf(stderr, "psg_run: %s: --resume needs the xHeI and xHeII blocks\n", snap_path);
			return 2;
		}
		for (size_t i = 0; i < n; i++) {
			lamHeI[i] = (double)xHeI[i];
			lamHeII[i] = (double)xHeII[i];
		}
		free(xHeI);
		free(xHeII);
	}

	/* units and tables (config.c defaults, cosmology.h from the file) */
	psg_unit_params up = {snap.h > 0 ? snap.h : 0.72, hmf, 3.0835455558318480e21, 1.9847005219450705e43,
			3.08568025e16};
	psg_units u;
	psg_rate_table ar;
	psg_xs_table xs;
	static double kernel[4096];
	int nk = 0;
	if (psg_units_init(&up, &u) != PSG_OK || psg_rate_table_load(rates_path, &u, &ar) != PSG_OK ||
			psg_xs_table_build(&u, &xs) != PSG_OK || psg_kernel_table_load(kernel_path, kernel, 4096, &nk) != PSG_OK) {
		fprintf(stderr, "psg_run: cannot build the tables from %s and %s\n", rates_path, kernel_path);
		return 2;
	}

	/* the device path */
	psg_context *ctx = NULL;
	int rc = psg_create(&ctx, (int)device);
	if (rc != PSG_OK) return lib_fail(ctx, rc, "psg_create (no usable GPU?)");
	const psg_flags fl = {isothermal, 1, hmf >= 1.0, 0, 0, 0};
	if ((rc = psg_set_physics(ctx, &u, &ar, &xs, kernel, nk, &fl)) != PSG_OK) return lib_fail(ctx, rc, "psg_set_physics");
	const psg_particles p = {n, pos, mass, sml, rho, ie, xHI, ye, NULL, snap.boxsize};
	if ((rc = psg_load_particles(ctx, &p)) != PSG_OK) return lib_fail(ctx, rc, "psg_load_particles");
	if (lamHeI && (rc = psg_set_he_state(ctx, lamHeI, lamHeII, NULL, NULL)) != PSG_OK)
		return lib_fail(ctx, rc, "psg_set_he_state");
	if ((rc = psg_build_tree(ctx, (int)ppc)) != PSG_OK) return lib_fail(ctx, rc, "psg_build_tree");

	/* point sources of one spectrum, constant luminosity */
	psg_source *srcs = calloc(nsrc, sizeof(psg_source));
	const int64_t hist_tick = 0;
	if (!srcs) return 2;
	for (size_t i = 0; i < nsrc; i++) {
		srcs[i].type = PSG_SRC_POINT;
		srcs[i].specid = 0;
		for (int k = 0; k < 3; k++) srcs[i].pos[k] = src_pos[3 * i + k];
		srcs[i].ticks = &hist_tick;
		srcs[i].ngamma_dot = &ngammas[i];
		srcs[i].nhist = 1;
		srcs[i].lastemit = 0;
	}
	double eng[8] = {energy_ev * u.EV}, weight[8] = {1.0};
	int nline = 1;
	if (bb_T > 0) {
		/* photon numbers of B_nu / (h nu) over log-spaced bins of 1-10 Ry,
		 * each line at the bin's geometric centre */
		const double kT = u.BOLTZMANN * bb_T;
		nline = 8;
		for (int k = 0; k < nline; k++) {
			const double e0 = u.RY_ENG * pow(10.0, (double)k / nline), e1 = u.RY_ENG * pow(10.0, (double)(k + 1) / nline);
			eng[k] = sqrt(e0 * e1);
			weight[k] = eng[k] * eng[k] / expm1(eng[k] / kT) * (e1 - e0);
		}
	}
	const psg_spectrum spec = {eng, weight, nline};
	if ((rc = psg_set_sources(ctx, srcs, (int)nsrc, &spec, 1, seed)) != PSG_OK) return lib_fail(ctx, rc, "psg_set_sources");

	/* the ticks */
	const double tick_time = myr * u.MYR / (double)nticks;
	double hits = 0.0, saturated = 0.0;
	const double t0 = now_s();
	for (long long t = 1; t <= nticks; t += batch) {
		const long long k = (t + batch - 1 <= nticks) ? batch : nticks - t + 1;
		psg_tick_stats st;
		if ((rc = psg_run_ticks_emit(ctx, (size_t)nray, (size_t)k, t, tick_time, &st)) != PSG_OK)
			return lib_fail(ctx, rc, "psg_run_ticks_emit");
		hits += st.hits;
		saturated += st.saturated;
	}
	const double secs = now_s() - t0;

	/* the epoch's output: state from the device; constants, ids and sources
	 * from the input */
	if ((rc = psg_write_output(ctx, out_path, &snap)) != PSG_OK) return lib_fail(ctx, rc, "psg_write_output");
	printf("psg_run: %zu particles, %zu sources, %lld ticks of %lld rays: %.6g hits (%.6g capped) in %.3f s, "
			"%.4g hits/s\n", n, nsrc, nticks, nray, hits, saturated, secs, secs > 0 ? hits / secs : 0.0);
	psg_destroy(ctx);
	psg_rate_table_free(&ar);
	psg_xs_table_free(&xs);
	free(srcs);
	free(pos); free(mass); free(sml); free(rho); free(ie); free(xHI); free(ye); free(src_pos); free(id); free(ngammas);
	free(lamHeI); free(lamHeII);
	return 0;
}
