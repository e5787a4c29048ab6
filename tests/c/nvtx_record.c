/* NVTX injection library for tests/test_tracing.py: loaded by NVTX v3 when
 * NVTX_INJECTION64_PATH names it, it appends every nvtxRangePushA ("push
 * <name>") and nvtxRangePop ("pop") of the process to the file named by
 * MBD_NVTX_RECORD, so that a test can see the ranges a call opens and closes
 * without a profiler. */
#include <stdio.h>
#include <stdlib.h>

#include <nvtx3/nvToolsExt.h>

static void put(const char* what, const char* name) {
    const char* path = getenv("MBD_NVTX_RECORD");
    FILE* f = path ? fopen(path, "a") : NULL;
    if (!f) return;
    if (name) fprintf(f, "%s %s\n", what, name);
    else fprintf(f, "%s\n", what);
    fclose(f);
}

static int range_push_a(const char* message) {
    put("push", message);
    return 0;
}

static int range_pop(void) {
    put("pop", NULL);
    return 0;
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_export_table) {
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get_export_table(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable table = NULL;
    unsigned int size = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size) || !table) return 0;
    if (size <= NVTX_CBID_CORE_RangePop) return 0;
    *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)range_push_a;
    *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)range_pop;
    return 1;
}
