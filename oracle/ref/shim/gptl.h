/* No-op GPTL timers for the host build of the reference drop-in (TEST INFRASTRUCTURE ONLY). */
#ifndef UWREF_GPTL_SHIM_H
#define UWREF_GPTL_SHIM_H
static inline int GPTLinitialize(void) { return 0; }
static inline int GPTLstart(const char *n) { (void)n; return 0; }
static inline int GPTLstop(const char *n) { (void)n; return 0; }
static inline int GPTLpr(int n) { (void)n; return 0; }
static inline int GPTLfinalize(void) { return 0; }
#endif
