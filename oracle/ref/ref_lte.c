/* The reference's LTE recombination spectrum, lte.c, compiled from the
 * reference tree inside this harness unit so that its tables (static in
 * lte.c) can be read back: lte_fill() lte.c:46-72 and lte_gen_freq()
 * lte.c:36-44 for the three species. Test infrastructure only. */
#include "lte.c"

void ref_lte_init(void) { lte_init(); }

/* Energies and weights of row `row` (log T = 3 + row*7/128) of table id
 * (0 HI, 1 HeI, 2 HeII); returns the number of energies (1024). */
int ref_lte_row(int id, int row, double *freq, double *weight) {
	const gsl_ran_discrete_t *g = lte[id].dist[row];
	for (size_t j = 0; j < lte[id].Nfreq; j++) {
		freq[j] = lte[id].freq[j];
		weight[j] = g->P[j];
	}
	return (int)lte[id].Nfreq;
}

/* lte_gen_freq() of table id with LTE on, its draw made at uniform u. */
double ref_lte_gen_freq(int id, double logT, double u) {
	const int saved = CFG_DISABLE_LTE;
	CFG_DISABLE_LTE = 0;
	oracle_shim_set_uniform(u);
	const double f = lte_gen_freq(id, logT);
	CFG_DISABLE_LTE = saved;
	return f;
}
