/* TEST INFRASTRUCTURE ONLY: stand-in for the PDI data interface of the reference's
 * writer.  pdi_shim.cpp records the layout metadata exposed at start-up and, on
 * the checkpoint event, writes the exposed host state (and time, step, step
 * size, WENO flags) to a raw file next to the .h5 name the reference chose. */
#ifndef KFVM_REFSHIM_PDI_H
#define KFVM_REFSHIM_PDI_H
#include "paraconf.h"
typedef enum { PDI_NONE = 0, PDI_IN = 1, PDI_OUT = 2, PDI_INOUT = 3 } PDI_inout_t;
typedef int PDI_status_t;
PDI_status_t PDI_init(PC_tree_t conf);
PDI_status_t PDI_finalize(void);
PDI_status_t PDI_multi_expose(const char *event_name, const char *name, const void *data,
                              PDI_inout_t access, ...);
#endif
