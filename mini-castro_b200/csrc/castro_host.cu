// castro_host.cu -- library state: error reporting, stream, network, the
// Helmholtz table (eos_init, Source/eos.F90:580-734) and the problem
// constants of initdata (Source/Prob.F90:11-15).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "castro_common.cuh"
#include "castro_table.h"
#include "../../include/castro_b200.h"

namespace castro {

// constant upload hooks of the other translation units
void upload_constants_abi(const EosTableDev& e, const NetworkDev& n);
void upload_constants_sim(const EosTableDev& e, const NetworkDev& n);
void upload_constants_adj(const EosTableDev& e, const NetworkDev& n);

namespace {
std::mutex g_mu;
int g_err = 0;
std::string g_errmsg;
cudaStream_t g_stream = 0;

NetworkDev g_net;
bool g_net_set = false;

bool g_table = false;
double* d_node = nullptr;
double* d_trow = nullptr;
double* d_drow = nullptr;
unsigned long long* d_fail = nullptr;
EosTableDev g_eos;

castro_problem g_prob;
bool g_prob_set = false;

// The packed node table (the 13 tables the hydro reads, 13.9 MB) is kept in L2
// by a persisting access-policy window on every sim's streams: between two
// EOS kernels each step streams gigabytes of face states and fluxes through
// L2, which would otherwise evict it.  The set-aside is this process's (it ends
// with the CUDA context) and is put back by eos_finalize.
bool g_l2_window = true;
// batched sims created afterwards run riemann2 + riemann3 as one column-tile kernel (2 species)
bool g_column_tiles = false;
size_t g_table_bytes = 0;
size_t g_l2_prev_limit = 0;
bool g_l2_limit_set = false;

void set_l2_limit()
{
    int dev = 0;
    cudaDeviceProp pr;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess) return;
    if (pr.persistingL2CacheMaxSize <= 0 || g_table_bytes == 0) return;
    if (!g_l2_limit_set && cudaDeviceGetLimit(&g_l2_prev_limit, cudaLimitPersistingL2CacheSize) != cudaSuccess) return;
    size_t want = g_table_bytes < (size_t)pr.persistingL2CacheMaxSize ? g_table_bytes : (size_t)pr.persistingL2CacheMaxSize;
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess) g_l2_limit_set = true;
    cudaGetLastError();
}

void restore_l2_limit()
{
    if (!g_l2_limit_set) return;
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, g_l2_prev_limit);
    cudaGetLastError();
    g_l2_limit_set = false;
}

void default_network()
{
    static const double a13[13] = {4., 12., 16., 20., 24., 28., 32., 36., 40., 44., 48., 52., 56.};
    static const double z13[13] = {2., 6., 8., 10., 12., 14., 16., 18., 20., 22., 24., 26., 28.};
    const int mfp = g_net.mom_flux_p, coul = g_net.coulomb;   // options, not part of the network
    memset(&g_net, 0, sizeof g_net);
    g_net.mom_flux_p = mfp;
    g_net.coulomb = coul;
    g_net.nspec = 13;
    for (int n = 0; n < 13; ++n) {
        g_net.aion[n] = a13[n];
        g_net.zion[n] = z13[n];
        g_net.aion_inv[n] = 1.0 / a13[n];
    }
    g_net_set = true;
}

void upload_all()
{
    if (!g_net_set) default_network();
    upload_constants_abi(g_eos, g_net);
    upload_constants_sim(g_eos, g_net);
    upload_constants_adj(g_eos, g_net);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) set_error(CASTRO_ERR_CUDA, cudaGetErrorString(e));
}

}  // namespace

void set_error(int code, const char* what)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_err == 0) {
        g_err = code;
        g_errmsg = what ? what : "";
    }
}
cudaStream_t stream() { return g_stream; }
bool table_ready() { return g_table; }
int nspec() { return g_net_set ? g_net.nspec : 13; }
const castro_problem& problem()
{
    if (!g_prob_set) {
        castro_problem_defaults(&g_prob);
        g_prob_set = true;
    }
    return g_prob;
}
const NetworkDev& network_host()
{
    if (!g_net_set) default_network();
    return g_net;
}
unsigned long long* eos_fail_counter() { return d_fail; }
bool coulomb_on() { return g_net.coulomb != 0; }
bool column_tiles_on() { return g_column_tiles; }

// the table's window on stream st (or no window, when it is switched off)
void apply_table_l2_window(cudaStream_t st)
{
    cudaStreamAttrValue v;
    memset(&v, 0, sizeof v);
    if (g_l2_window && g_table && d_node && g_l2_limit_set) {
        int dev = 0;
        cudaDeviceProp pr;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess) return;
        size_t n = g_table_bytes < (size_t)pr.accessPolicyMaxWindowSize ? g_table_bytes : (size_t)pr.accessPolicyMaxWindowSize;
        v.accessPolicyWindow.base_ptr = d_node;
        v.accessPolicyWindow.num_bytes = n;
        v.accessPolicyWindow.hitRatio = 1.0f;
        v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    }
    cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaGetLastError();
}

}  // namespace castro

using namespace castro;

extern "C" {

int castro_last_error(void) { std::lock_guard<std::mutex> lk(g_mu); return g_err; }
void castro_clear_error(void) { std::lock_guard<std::mutex> lk(g_mu); g_err = 0; g_errmsg.clear(); }
const char* castro_error_string(void) { std::lock_guard<std::mutex> lk(g_mu); return g_errmsg.c_str(); }
int castro_version(void) { return 100; }
void castro_set_stream(void* s) { g_stream = (cudaStream_t)s; }
void* castro_get_stream(void) { return (void*)g_stream; }
int castro_exact_build(void)
{
#ifdef CASTRO_EXACT
    return 1;
#else
    return 0;
#endif
}

void network_init(void)
{
    default_network();
    if (g_table) upload_all();
}

void network_finalize(void) {}

int castro_network_init(int ns, const double* aion, const double* zion)
{
    if (ns != 2 && ns != 13) {
        set_error(CASTRO_ERR_NSPEC, "castro_network_init: nspec must be 2 or 13");
        return CASTRO_ERR_NSPEC;
    }
    const int mfp = g_net.mom_flux_p, coul = g_net.coulomb;   // options, not part of the network
    memset(&g_net, 0, sizeof g_net);
    g_net.mom_flux_p = mfp;
    g_net.coulomb = coul;
    g_net.nspec = ns;
    for (int n = 0; n < ns; ++n) {
        g_net.aion[n] = aion[n];
        g_net.zion[n] = zion[n];
        g_net.aion_inv[n] = 1.0 / aion[n];
    }
    g_net_set = true;
    if (g_table) upload_all();
    return CASTRO_OK;
}

int castro_nspec(void) { return nspec(); }

void castro_set_table_l2_window(int on) { g_l2_window = on != 0; }
void castro_set_column_tiles(int on) { g_column_tiles = on != 0; }
int castro_column_tiles(void) { return g_column_tiles ? 1 : 0; }

void castro_set_momentum_flux_pressure(int on)
{
    g_net.mom_flux_p = on != 0;
    if (!g_table) return;   // uploaded with the table
    // kernels already queued on any stream read the constants when they run:
    // let them finish under the old value first
    cudaDeviceSynchronize();
    upload_all();
}

int castro_momentum_flux_pressure(void) { return g_net.mom_flux_p; }

void castro_set_coulomb_corrections(int on)
{
    g_net.coulomb = on != 0;
    if (!g_table) return;   // uploaded with the table
    cudaDeviceSynchronize();   // queued kernels finish under the old value
    upload_all();
}

int castro_coulomb_corrections(void) { return g_net.coulomb; }

int castro_eos_init_path(const char* path)
{
    NvtxRange r("eos_init");
    HostTable T;
    int rc = read_helm_table(path, T);
    if (rc == 1) {
        std::string m = std::string("eos_init: cannot open ") + path;
        set_error(CASTRO_ERR_TABLE_IO, m.c_str());
        return CASTRO_ERR_TABLE_IO;
    }
    if (rc != 0) {
        set_error(CASTRO_ERR_TABLE_IO, "eos_init: helm_table.dat is truncated or malformed");
        return CASTRO_ERR_TABLE_IO;
    }
    eos_finalize();
    cudaError_t e = cudaMalloc(&d_node, T.node.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_trow, T.trow.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_drow, T.drow.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_fail, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemcpy(d_node, T.node.data(), T.node.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_trow, T.trow.data(), T.trow.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_drow, T.drow.data(), T.drow.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_fail, 0, sizeof(unsigned long long));
    if (e != cudaSuccess) {
        set_error(CASTRO_ERR_CUDA, cudaGetErrorString(e));
        return CASTRO_ERR_CUDA;
    }
    g_table_bytes = T.node.size() * sizeof(double);
    set_l2_limit();
    g_eos = T.consts;
    g_eos.node = d_node;
    g_eos.trow = d_trow;
    g_eos.drow = d_drow;
    g_eos.fail_count = d_fail;
    g_table = true;
    upload_all();
    return castro_last_error() == 0 ? CASTRO_OK : castro_last_error();
}

void eos_init(void)
{
    const char* p = getenv("CASTRO_HELM_TABLE");
    castro_eos_init_path(p && *p ? p : "helm_table.dat");
}

void eos_finalize(void)
{
    restore_l2_limit();
    if (d_node) cudaFree(d_node);
    if (d_trow) cudaFree(d_trow);
    if (d_drow) cudaFree(d_drow);
    if (d_fail) cudaFree(d_fail);
    d_node = d_trow = d_drow = nullptr;
    d_fail = nullptr;
    g_table = false;
}

void castro_problem_defaults(castro_problem* p)
{
    memset(p, 0, sizeof *p);
    p->ambient_from_T = 0;
    p->dens_ambient = 1.e4;
    p->p_ambient = 1.e21;
    p->T_ambient = 1.e6;
    p->exp_energy = 1.e52;
    p->r_init = 1.25e8;
    p->nsub = 10;
    p->X[0] = 1.0;
    p->T_init = 1.e9;
}

int castro_set_problem(const castro_problem* p)
{
    if (!p || p->nsub < 1 || !(p->dens_ambient > 0.0)) {
        set_error(CASTRO_ERR_ARG, "castro_set_problem: invalid problem");
        return CASTRO_ERR_ARG;
    }
    g_prob = *p;
    g_prob_set = true;
    return CASTRO_OK;
}

}  // extern "C"
