/* Stand-in for psrdada's dada_def.h (not vendored); nothing from it is used
 * beyond the include.  Project-written. */
#ifndef REF_SHIM_DADA_DEF_H
#define REF_SHIM_DADA_DEF_H
#endif
