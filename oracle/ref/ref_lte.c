/* The reference's LTE recombination spectrum, lte.c, compiled from the
 * reference tree inside this harness unit so that its tables (static in
 * lte.c) can be read back: lte_fill() lte.c:46-72 and lte_gen_freq()
 * lte.c:36-44 for hydrogen. Test infrastructure only. */
#include "lte.c"

void ref_lte_init(void) { lte_init(); }

/* Energies and weights of row `row` (log T = 3 + row*7/128) of the HI
 * table; returns the number of energies (1024). */
int ref_lte_row(int row, double *freq, double *weight) {
	const gsl_ran_discrete_t *g = lte[LTE_FREQ_HI].dist[row];
	for (size_t j = 0; j < lte[LTE_FREQ_HI].Nfreq; j++) {
		freq[j] = lte[LTE_FREQ_HI].freq[j];
		weight[j] = g->P[j];
	}
	return (int)lte[LTE_FREQ_HI].Nfreq;
}

/* lte_gen_freq() with LTE on, its draw made at uniform u. */
double ref_lte_gen_freq(double logT, double u) {
	const int saved = CFG_DISABLE_LTE;
	CFG_DISABLE_LTE = 0;
	oracle_shim_set_uniform(u);
	const double f = lte_gen_freq(LTE_FREQ_HI, logT);
	CFG_DISABLE_LTE = saved;
	return f;
}
