/* psphray-format snapshots: the output of psystem_write_output()
 * (psystem.c:598-690) and the input a run resumes from.
 *
 * The format is the reference's (reader-psphray.inc, generated by gen.py):
 * a 256-byte header packed to 4-byte alignment, then the blocks in a fixed
 * order, each present block as a 4-byte size, the data, the size again.
 * A block is present when its length times its item size is not zero; its
 * length follows from the header's particle counts and flags:
 *
 *   id  block        item  length
 *   0   header       256   1
 *   1   pos          12    N0 + N4 + N5      (gas, then stars, then sources)
 *   2   id           8     N0 + N4 + N5
 *   3   mass         4     N0 + N4 + N5
 *   4-8 ie rho ye xHI sml   4     N0
 *   9   Hmf          4     N0 if flag_Hmf        10 Hemf  if flag_Hemf
 *   11  xHeI, 12 xHeII 4   N0 if flag_Helium     13 gammaHI if flag_gammaHI
 *   14  HIa_cloudy   4     N0 if flag_cloudy     15 eos     if flag_eos
 *   16  lasthit      8     N0                    17 hits (4) N0
 *   18  sft          4     N4                    19 ngammas (8), 20 spec (8) N5
 *
 * The writer fills the header as psystem_write_output() does (helium and
 * gammaHI blocks on, the reference's default flags otherwise) and writes one
 * file; the reader takes any single file of this format.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "psg.h"

enum { B_HEADER, B_POS, B_ID, B_MASS, B_IE, B_RHO, B_YE, B_XHI, B_SML, B_HMF, B_HEMF, B_XHEI, B_XHEII,
	B_GAMMAHI, B_CLOUDY, B_EOS, B_LASTHIT, B_HITS, B_SFT, B_NGAMMAS, B_SPEC, B_NBLOCKS };

static const size_t kItem[B_NBLOCKS] = {256, 12, 8, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 8, 4, 4, 8, 8};

/* header field offsets (the 4-byte-packed layout of reader-psphray.inc) */
enum { H_N = 0, H_MASS = 24, H_TIME = 72, H_REDSHIFT = 80, H_FLAG_SFR = 88, H_FLAG_FEEDBACK = 92,
	H_NTOT_LOW = 96, H_FLAG_COOL = 120, H_NFILES = 124, H_BOXSIZE = 128, H_OMEGAM = 136, H_OMEGAL = 144,
	H_H = 152, H_FLAG_SFT = 160, H_FLAG_MET = 164, H_NTOT_HIGH = 168, H_FLAG_ENTROPY = 192, H_OMEGAB = 196,
	H_NRAYS = 204, H_FLAG_HMF = 212, H_FLAG_HEMF = 216, H_FLAG_HELIUM = 220, H_FLAG_GAMMAHI = 224,
	H_FLAG_CLOUDY = 228, H_FLAG_EOS = 232 };

static void put_u32(unsigned char *h, int off, uint32_t v) { memcpy(h + off, &v, 4); }
static void put_i32(unsigned char *h, int off, int32_t v) { memcpy(h + off, &v, 4); }
static void put_f64(unsigned char *h, int off, double v) { memcpy(h + off, &v, 8); }
static uint32_t get_u32(const unsigned char *h, int off) { uint32_t v; memcpy(&v, h + off, 4); return v; }
static int32_t get_i32(const unsigned char *h, int off) { int32_t v; memcpy(&v, h + off, 4); return v; }
static double get_f64(const unsigned char *h, int off) { double v; memcpy(&v, h + off, 8); return v; }

/* block lengths (items) from a header */
static void lengths(const unsigned char *h, size_t len[B_NBLOCKS]) {
	const size_t n0 = get_u32(h, H_N + 0), n4 = get_u32(h, H_N + 16), n5 = get_u32(h, H_N + 20);
	const int hmf = get_i32(h, H_FLAG_HMF), hemf = get_i32(h, H_FLAG_HEMF), he = get_i32(h, H_FLAG_HELIUM);
	const int gam = get_i32(h, H_FLAG_GAMMAHI), cl = get_i32(h, H_FLAG_CLOUDY), eos = get_i32(h, H_FLAG_EOS);
	len[B_HEADER] = 1;
	len[B_POS] = len[B_ID] = len[B_MASS] = n0 + n4 + n5;
	len[B_IE] = len[B_RHO] = len[B_YE] = len[B_XHI] = len[B_SML] = n0;
	len[B_HMF] = hmf ? n0 : 0;
	len[B_HEMF] = hemf ? n0 : 0;
	len[B_XHEI] = len[B_XHEII] = he ? n0 : 0;
	len[B_GAMMAHI] = gam ? n0 : 0;
	len[B_CLOUDY] = cl ? n0 : 0;
	len[B_EOS] = eos ? n0 : 0;
	len[B_LASTHIT] = len[B_HITS] = n0;
	len[B_SFT] = n4;
	len[B_NGAMMAS] = len[B_SPEC] = n5;
}

static void offsets(const size_t len[B_NBLOCKS], size_t off[B_NBLOCKS]) {
	size_t o = 0;
	for (int b = 0; b < B_NBLOCKS; b++) {
		off[b] = o;
		const size_t bytes = len[b] * kItem[b];
		if (bytes) o += bytes + 8;
	}
}

/* one block: size marker, the gas part (or zeros), the rest zeros, marker */
static int write_block(FILE *fp, int b, const size_t len[B_NBLOCKS], const void *data, size_t ndata,
		const void *tail, size_t ntail) {
	const size_t bytes = len[b] * kItem[b];
	if (!bytes) return PSG_OK;
	if (bytes > 0x7fffffffu) return PSG_E_OVERFLOW;       /* the size markers are 32-bit */
	const int32_t marker = (int32_t)bytes;
	if (fwrite(&marker, 4, 1, fp) != 1) return PSG_E_IO;
	size_t done = 0;
	static const unsigned char zeros[4096];
	if (data && ndata) {
		if (fwrite(data, kItem[b], ndata, fp) != ndata) return PSG_E_IO;
		done += ndata * kItem[b];
	}
	/* a gap before the tail (the parts a writer leaves unset are zero) */
	const size_t tail_at = tail ? bytes - ntail * kItem[b] : bytes;
	while (done < tail_at) {
		const size_t k = tail_at - done < sizeof(zeros) ? tail_at - done : sizeof(zeros);
		if (fwrite(zeros, 1, k, fp) != k) return PSG_E_IO;
		done += k;
	}
	if (tail && ntail) {
		if (fwrite(tail, kItem[b], ntail, fp) != ntail) return PSG_E_IO;
		done += ntail * kItem[b];
	}
	if (fwrite(&marker, 4, 1, fp) != 1) return PSG_E_IO;
	return PSG_OK;
}

int psg_snapshot_write(const char *filename, const psg_snapshot *s) {
	if (!filename || !s) return PSG_E_INVAL;
	if (s->ngas > 0xffffffffu || s->nsrc > 0xffffffffu) return PSG_E_OVERFLOW;
	unsigned char h[256];
	memset(h, 0, sizeof h);
	put_u32(h, H_N + 0, (uint32_t)s->ngas);
	put_u32(h, H_N + 20, (uint32_t)s->nsrc);
	put_u32(h, H_NTOT_LOW + 0, (uint32_t)s->ngas);
	put_u32(h, H_NTOT_LOW + 20, (uint32_t)s->nsrc);
	put_f64(h, H_TIME, s->time);
	put_f64(h, H_REDSHIFT, s->redshift);
	put_f64(h, H_BOXSIZE, s->boxsize);
	put_f64(h, H_OMEGAM, s->OmegaM);
	put_f64(h, H_OMEGAL, s->OmegaL);
	put_f64(h, H_OMEGAB, s->OmegaB);
	put_f64(h, H_H, s->h);
	put_i32(h, H_NFILES, 1);
	/* the reference's default header (_def_header) with helium and gammaHI on */
	put_i32(h, H_FLAG_SFR, 1);
	put_i32(h, H_FLAG_FEEDBACK, 1);
	put_i32(h, H_FLAG_COOL, 1);
	put_i32(h, H_FLAG_SFT, 1);
	put_i32(h, H_FLAG_MET, 1);
	put_i32(h, H_FLAG_HELIUM, 1);
	put_i32(h, H_FLAG_GAMMAHI, 1);
	size_t len[B_NBLOCKS];
	lengths(h, len);
	FILE *fp = fopen(filename, "wb");
	if (!fp) return PSG_E_IO;
	const size_t n = s->ngas, ns = s->nsrc;
	int rc = write_block(fp, B_HEADER, len, h, 1, NULL, 0);
	if (!rc) rc = write_block(fp, B_POS, len, s->pos, s->pos ? n : 0, s->src_pos, s->src_pos ? ns : 0);
	if (!rc) rc = write_block(fp, B_ID, len, s->id, s->id ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_MASS, len, s->mass, s->mass ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_IE, len, s->ie, s->ie ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_RHO, len, s->rho, s->rho ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_YE, len, s->ye, s->ye ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_XHI, len, s->xHI, s->xHI ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_SML, len, s->sml, s->sml ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_XHEI, len, s->xHeI, s->xHeI ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_XHEII, len, s->xHeII, s->xHeII ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_GAMMAHI, len, s->gammaHI, s->gammaHI ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_LASTHIT, len, s->lasthit, s->lasthit ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_HITS, len, s->hits, s->hits ? n : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_NGAMMAS, len, s->ngammas, s->ngammas ? ns : 0, NULL, 0);
	if (!rc) rc = write_block(fp, B_SPEC, len, NULL, 0, NULL, 0);
	if (fclose(fp) != 0 && !rc) rc = PSG_E_IO;
	return rc;
}

static int read_header(FILE *fp, unsigned char h[256]) {
	int32_t m0 = 0, m1 = 0;
	if (fread(&m0, 4, 1, fp) != 1 || m0 != 256 || fread(h, 1, 256, fp) != 256 || fread(&m1, 4, 1, fp) != 1 ||
			m1 != 256)
		return PSG_E_IO;
	return PSG_OK;
}

int psg_snapshot_read_header(const char *filename, psg_snapshot *s) {
	if (!filename || !s) return PSG_E_INVAL;
	FILE *fp = fopen(filename, "rb");
	if (!fp) return PSG_E_IO;
	unsigned char h[256];
	const int rc = read_header(fp, h);
	fclose(fp);
	if (rc) return rc;
	s->ngas = get_u32(h, H_N + 0);
	s->nsrc = get_u32(h, H_N + 20);
	s->time = get_f64(h, H_TIME);
	s->redshift = get_f64(h, H_REDSHIFT);
	s->boxsize = get_f64(h, H_BOXSIZE);
	s->OmegaM = get_f64(h, H_OMEGAM);
	s->OmegaL = get_f64(h, H_OMEGAL);
	s->OmegaB = get_f64(h, H_OMEGAB);
	s->h = get_f64(h, H_H);
	return PSG_OK;
}

/* reads `count` items from position `start` of block b into dst */
static int read_block(FILE *fp, int b, const size_t len[B_NBLOCKS], const size_t off[B_NBLOCKS], size_t start,
		size_t count, void *dst) {
	if (!dst || !count) return PSG_OK;
	const size_t bytes = len[b] * kItem[b];
	if (!bytes || start + count > len[b]) return PSG_E_IO;     /* block absent from this file */
	int32_t m0 = 0, m1 = 0;
	if (fseek(fp, (long)off[b], SEEK_SET) != 0 || fread(&m0, 4, 1, fp) != 1 || (size_t)(uint32_t)m0 != bytes)
		return PSG_E_IO;
	if (fseek(fp, (long)(start * kItem[b]), SEEK_CUR) != 0 || fread(dst, kItem[b], count, fp) != count)
		return PSG_E_IO;
	if (fseek(fp, (long)(off[b] + 4 + bytes), SEEK_SET) != 0 || fread(&m1, 4, 1, fp) != 1 || m1 != m0)
		return PSG_E_IO;
	return PSG_OK;
}

int psg_snapshot_read(const char *filename, psg_snapshot *s) {
	if (!filename || !s) return PSG_E_INVAL;
	FILE *fp = fopen(filename, "rb");
	if (!fp) return PSG_E_IO;
	unsigned char h[256];
	int rc = read_header(fp, h);
	if (rc) { fclose(fp); return rc; }
	size_t len[B_NBLOCKS], off[B_NBLOCKS];
	lengths(h, len);
	offsets(len, off);
	const size_t n = get_u32(h, H_N + 0), n4 = get_u32(h, H_N + 16), ns = get_u32(h, H_N + 20);
	if (n != s->ngas || ns != s->nsrc) { fclose(fp); return PSG_E_INVAL; }
	rc = read_block(fp, B_POS, len, off, 0, n, s->pos);
	if (!rc) rc = read_block(fp, B_POS, len, off, n + n4, ns, s->src_pos);
	if (!rc) rc = read_block(fp, B_ID, len, off, 0, n, s->id);
	if (!rc) rc = read_block(fp, B_MASS, len, off, 0, n, s->mass);
	if (!rc) rc = read_block(fp, B_IE, len, off, 0, n, s->ie);
	if (!rc) rc = read_block(fp, B_RHO, len, off, 0, n, s->rho);
	if (!rc) rc = read_block(fp, B_YE, len, off, 0, n, s->ye);
	if (!rc) rc = read_block(fp, B_XHI, len, off, 0, n, s->xHI);
	if (!rc) rc = read_block(fp, B_SML, len, off, 0, n, s->sml);
	if (!rc) rc = read_block(fp, B_XHEI, len, off, 0, n, s->xHeI);
	if (!rc) rc = read_block(fp, B_XHEII, len, off, 0, n, s->xHeII);
	if (!rc) rc = read_block(fp, B_GAMMAHI, len, off, 0, n, s->gammaHI);
	if (!rc) rc = read_block(fp, B_LASTHIT, len, off, 0, n, s->lasthit);
	if (!rc) rc = read_block(fp, B_HITS, len, off, 0, n, s->hits);
	if (!rc) rc = read_block(fp, B_NGAMMAS, len, off, 0, ns, s->ngammas);
	fclose(fp);
	return rc;
}
