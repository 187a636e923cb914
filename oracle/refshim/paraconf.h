/* TEST INFRASTRUCTURE ONLY: the paraconf calls of the reference's main(), with no
 * YAML behind them (the PDI stand-in needs no configuration). */
#ifndef KFVM_REFSHIM_PARACONF_H
#define KFVM_REFSHIM_PARACONF_H
typedef struct {
  int status;
} PC_tree_t;
static inline PC_tree_t PC_parse_path(const char *) { PC_tree_t t = {0}; return t; }
static inline PC_tree_t PC_get(PC_tree_t t, const char *) { return t; }
static inline int PC_tree_destroy(PC_tree_t *) { return 0; }
#endif
