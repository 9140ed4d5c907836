/* Test infrastructure: the reference's own snapshot reader (src/reader.c,
 * src/reader-psphray.c) behind one plain function, so that the tests can
 * read files written by psg_snapshot_write with the reference's code.
 *
 * Called once with NULL arrays for the counts and constants, then with
 * arrays of those sizes. */
#include <stddef.h>
#include <stdint.h>

#include "reader.h"

int refrd_read(const char *filename, size_t *ngas, size_t *nsrc, double consts[7], float *pos, int64_t *id,
		float *mass, float *ie, float *rho, float *ye, float *xHI, float *sml, float *xHeI, float *xHeII,
		float *gammaHI, int64_t *lasthit, int32_t *hits, float *src_pos, double *ngammas) {
	Reader *r = reader_new("psphray");
	reader_open(r, filename);
	ReaderConstants *c = reader_constants(r);
	*ngas = c->N[0];
	*nsrc = c->N[5];
	consts[0] = c->time;
	consts[1] = c->redshift;
	consts[2] = c->boxsize;
	consts[3] = c->OmegaM;
	consts[4] = c->OmegaL;
	consts[5] = c->OmegaB;
	consts[6] = c->h;
	if (pos) reader_read(r, "pos", 0, pos);
	if (id) reader_read(r, "id", 0, id);
	if (mass) reader_read(r, "mass", 0, mass);
	if (ie) reader_read(r, "ie", 0, ie);
	if (rho) reader_read(r, "rho", 0, rho);
	if (ye) reader_read(r, "ye", 0, ye);
	if (xHI) reader_read(r, "xHI", 0, xHI);
	if (sml) reader_read(r, "sml", 0, sml);
	if (xHeI) reader_read(r, "xHeI", 0, xHeI);
	if (xHeII) reader_read(r, "xHeII", 0, xHeII);
	if (gammaHI) reader_read(r, "gammaHI", 0, gammaHI);
	if (lasthit) reader_read(r, "lasthit", 0, lasthit);
	if (hits) reader_read(r, "hits", 0, hits);
	if (src_pos) reader_read(r, "pos", 5, src_pos);
	if (ngammas) reader_read(r, "ngammas", 5, ngammas);
	reader_close(r);
	reader_destroy(r);
	return 0;
}
