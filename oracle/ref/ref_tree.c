/* Second oracle harness unit: #includes the reference's src/raytrace.c (in
 * place of compiling it on its own) so that the octree pool `rt` built by
 * rt_switch_epoch() raytrace.c:41-151 can be read back cell by cell for the
 * tree-parity tests. Test infrastructure only. */
#include "raytrace.c"

size_t ref_tree_ncells(void) { return rt.pool_used; }
void ref_tree_cells(int64_t *head_par, int64_t *first_child, int64_t *parent,
		uint32_t *npar, float *bot, float *top) {
	for (intptr_t i = 0; i < rt.pool_used; i++) {
		head_par[i] = rt.pool[i].head_par;
		first_child[i] = rt.pool[i].first_child;
		parent[i] = rt.pool[i].parent;
		npar[i] = rt.pool[i].npar;
		for (int d = 0; d < 3; d++) {
			bot[3 * i + d] = rt.pool[i].bot[d];
			top[3 * i + d] = rt.pool[i].top[d];
		}
	}
}
void ref_tree_next(int64_t *next) {
	for (size_t i = 0; i < psys.npar; i++) next[i] = rt.next[i];
}

