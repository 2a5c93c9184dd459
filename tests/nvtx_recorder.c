/* nvtx_recorder.c -- a minimal NVTX injection library for the tracing test.
 *
 * NVTX3 loads the library named by NVTX_INJECTION64_PATH on the first NVTX
 * call of a process and calls its InitializeInjectionNvtx2, which may replace
 * entries of the per-module function tables.  This one replaces the domain
 * create / range push / range pop entries with functions that append one line
 * per call to the file named by LSVD_NVTX_LOG:
 *   "domain <name>", "push <message>", "pop".
 * Build: gcc -shared -fPIC -I<cuda>/include nvtx_recorder.c -o nvtx_recorder.so */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <nvtx3/nvToolsExt.h>

static FILE* g_log;

static void put(const char* what, const char* text) {
    if (!g_log) return;
    if (text) fprintf(g_log, "%s %s\n", what, text);
    else fprintf(g_log, "%s\n", what);
    fflush(g_log);
}

static nvtxDomainHandle_t NVTX_API rec_domain_create(const char* name) {
    put("domain", name);
    return (nvtxDomainHandle_t)(uintptr_t)1;
}

static int NVTX_API rec_push(nvtxDomainHandle_t d, const nvtxEventAttributes_t* a) {
    (void)d;
    put("push", a && a->messageType == NVTX_MESSAGE_TYPE_ASCII ? a->message.ascii : "?");
    return 0;
}

static int NVTX_API rec_pop(nvtxDomainHandle_t d) {
    (void)d;
    put("pop", NULL);
    return 0;
}

__attribute__((visibility("default"))) int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get) {
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable t = 0;
    unsigned int size = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE2, &t, &size) || !t ||
        size < NVTX_CBID_CORE2_DomainCreateA)
        return 0;
    *t[NVTX_CBID_CORE2_DomainCreateA] = (NvtxFunctionPointer)rec_domain_create;
    *t[NVTX_CBID_CORE2_DomainRangePushEx] = (NvtxFunctionPointer)rec_push;
    *t[NVTX_CBID_CORE2_DomainRangePop] = (NvtxFunctionPointer)rec_pop;
    if (!g_log) {
        const char* path = getenv("LSVD_NVTX_LOG");
        g_log = path ? fopen(path, "a") : NULL;
    }
    return 1;
}
