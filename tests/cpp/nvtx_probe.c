/* NVTX injection probe (test infrastructure): loaded by NVTX through
 * NVTX_INJECTION64_PATH, it records the name of every range pushed with
 * nvtxRangePushA, one per line, in the file named by MTB_NVTX_LOG.  Uses only
 * the injection interface declared in nvtx3/nvtxDetail/nvtxTypes.h. */
#include <stdio.h>
#include <stdlib.h>

#include <nvtx3/nvToolsExt.h>

static FILE *g_log;

static int probe_push(const char *message) {
    if (g_log) {
        fprintf(g_log, "push %s\n", message ? message : "");
        fflush(g_log);
    }
    return 0;
}

static int probe_pop(void) {
    if (g_log) {
        fprintf(g_log, "pop\n");
        fflush(g_log);
    }
    return 0;
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_table) {
    const char *path = getenv("MTB_NVTX_LOG");
    if (!path) return 0;
    g_log = fopen(path, "w");
    const NvtxExportTableCallbacks *cb = (const NvtxExportTableCallbacks *)get_table(NVTX_ETID_CALLBACKS);
    if (!cb || !g_log) return 0;
    NvtxFunctionTable table = 0;
    unsigned int size = 0;
    if (!cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size) || !table) return 0;
    if (size > NVTX_CBID_CORE_RangePushA) *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)probe_push;
    if (size > NVTX_CBID_CORE_RangePop) *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)probe_pop;
    return 1;
}
