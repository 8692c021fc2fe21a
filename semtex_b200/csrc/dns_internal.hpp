// The DNS handle (stx_dns) shared by the time stepper (dns.cu) and its
// discrete adjoint (adjoint.cu), and the step functions both use.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "kernels/exprprog.hpp"
#include "kernels/outflow.cuh"
#include "stx_internal.hpp"

struct stx_dns {
  using DeviceArena = stx::DeviceArena;
  using ExprOp = stx::ExprOp;
  stx_context* ctx = nullptr;
  int ncom = 0, ndim = 0, nord = 0, form = 1;
  double dt = 0, nu = 0, beta = 0, tol = 0;
  int step_max = 0;
  bool iterative = false;  // ITERATIVE: Jacobi-PCG velocity systems at every step
  bool mixed = false;      // STX_DNS_MIXED: mixed-precision steady velocity systems
  int step = 0;
  double time = 0;
  int toggle = 1;  // altSkewSymmetric's static switch (dns/nonlinear.cpp:254)
  std::string names;  // velocity components then pressure
  DeviceArena arena;
  size_t fsize = 0;  // doubles per field
  std::vector<double*> u;                 // [ncom+1] Domain fields (Fourier)
  std::vector<std::vector<double*>> Us, Uf;  // [nord][ncom]
  std::vector<double*> Up;                // [ncom] physical velocities
  double* tmp0 = nullptr;
  double* tmp1 = nullptr;
  double* tmp2 = nullptr;
  double* dsswork = nullptr;
  std::vector<stx_modal*> vsys;           // DIRECT velocity systems
  stx_modal* psys = nullptr;
  std::map<std::pair<char, int>, stx_modal*> pcg;  // temporary JACPCG systems
  std::vector<char> tdep;                 // per field: BCs depend on t
  std::vector<int> last_iters;
  // High-order pressure BCs: edge tables and the multi-level storage of u.n
  // and of the BC terms (BCmgr::_un / _hopbc), levels newest first and
  // rolled by pointer like rollv (src/sem.h:98-106).
  int nh = 0;
  const int* h_elmt = nullptr;
  const int* h_side = nullptr;
  const int* h_line = nullptr;
  const double* h_nx = nullptr;
  const double* h_ny = nullptr;
  std::vector<double*> un_lvl, hop_lvl;
  size_t hsize = 0;  // doubles per level
  // Computed outflow BCs <O> (outflow.cuh): edges, and the levels (newest
  // first, rolled by pointer) of the physical edge velocities, nu div u and
  // nu n.grad(u).n; o_fb holds KE* S0 of the step.
  stx::OutflowEdges oe{};
  std::vector<double*> o_uvw, o_divu, o_gradu;
  double* o_fb = nullptr;
  double o_iuzd = 0.0;  // 1 / U0Delta
  // 3/2-rule products (token DEALIAS, N_Z > 2): physical fields on nz32 =
  // 3 N_Z / 2 planes (AuxField::transform32, src/auxfield.cpp:1197-1258).
  int nz32 = 0;
  double* twiddle32 = nullptr;
  std::vector<double*> Up32;               // [ncom] padded physical velocities
  double* A32 = nullptr;                   // padded nonlinear terms
  double* B32 = nullptr;                   // padded z-derivative term (convective)
  double* C32 = nullptr;                   // padded product / z-derivative term (conservative)
  double* part = nullptr;                  // analysis partials: blocks x max(modes, 3)
  // Edges of the boundary group named "wall" (Field::normTraction /
  // tangTraction, src/field.cpp:392-458): element, side nodes in the side
  // traverse, unit outward normal and quadrature-weighted length per node,
  // and the per-edge sums of stx_dns_wall_forces.
  int nwall = 0;
  const int* w_elmt = nullptr;
  const int* w_node = nullptr;
  const double* w_nx = nullptr;
  const double* w_ny = nullptr;
  const double* w_area = nullptr;
  double* w_out = nullptr;
  int w_npad = 0;            // traction plane length: 3 np nwall rounded up to even
  double* w_buf = nullptr;   // [nz][w_npad] tractions (stx_dns_wall_traction)
  // History-point scratch (stx_dns_probe), grown on demand: per-point
  // weights, elements and results.
  void* probe_buf = nullptr;
  size_t probe_bytes = 0;
  // Steady steps replayed as a CUDA graph (token STX_DNS_GRAPH, default 1):
  // the steps from one pointer state back to the same state (the multi-level
  // storage rolls by pointer, the alternating form toggles) captured once.
  bool use_graph = true;
  cudaGraphExec_t gexec = nullptr;
  int gperiod = 0;
  std::vector<double*> gkey;  // pointer state the captured steps start from and return to
  int gtoggle = 0;
  int eager_steady = 0;       // steady steps run directly since the last restart
  long long graph_launches = 0;
  // Running averages (Statistics, src/statistics.cpp:94-466; token AVERAGE
  // 1 or 2): buffers named as the reference names them, in its order (the
  // sorted keys of its map): the raw fields held in Fourier space and, for
  // AVERAGE 2, the velocity products A = uu, B = uv, C = vv, D = uw, E = vw,
  // F = ww held in physical space.
  int avg_level = 0;
  int navg = 0;
  std::string avg_names;
  std::vector<double*> avg_buf;
  double* avg_work = nullptr;  // AVERAGE 3: seven work fields
  std::vector<double*> avg_alt; // the second set of averages (stx_dns_stats_swap)
  int navg_alt = 0;
  // Body forcing (<FORCE>; FieldForce and its classes, dns/fieldforce.cpp),
  // on the grid of the nonlinear products (nzl planes: N_Z, or 3 N_Z / 2
  // with DEALIAS).  Fields are device arrays of nzl planes, null when a term
  // is absent; time-dependent scalars are evaluated on the host each step.
  struct Force {
    bool on = false;        // FORCE section present
    bool physical = false;  // some physical-space term present
    bool tdep = false;      // some term changes from step to step
    double cst[3] = {0.0, 0.0, 0.0};  // ConstForce
    int nzl = 0;
    double dz = 0.0;
    double* x = nullptr;  // node coordinates [nplane]
    double* y = nullptr;
    double* mask = nullptr;  // SpongeForce
    double* uref[3] = {nullptr, nullptr, nullptr};
    int sponge_update = 0;
    ExprOp* mask_prog = nullptr;
    int nmask = 0;
    int coriolis = 0;  // CoriolisForce: 0 off, 1 steady, 2 unsteady
    std::string omega[3], domega[3];
    double m2o[3] = {0.0, 0.0, 0.0}, o[3] = {0.0, 0.0, 0.0}, mo[3] = {0.0, 0.0, 0.0},
           dodt[3] = {0.0, 0.0, 0.0};
    double* steady[3] = {nullptr, nullptr, nullptr};  // SteadyForce
    std::string alpha[3];                              // ModulatedForce
    double* moda[3] = {nullptr, nullptr, nullptr};
    ExprOp* st[3] = {nullptr, nullptr, nullptr};  // SpatioTemporalForce
    int nst[3] = {0, 0, 0};
    double* drag = nullptr;  // DragForce
    double* qbar[3] = {nullptr, nullptr, nullptr};  // SFDForce
    double chi = 0.0, rate = 0.0;
    bool sfd_started = false;
  } force;
};

namespace stx {

// Stiffly stable coefficients of orders 1..3 (alpha_0..alpha_J) and the
// matching extrapolation weights (src/integration.cpp:99-164).
extern const double kSS[4][4];
extern const double kEX[4][3];

// One time step of integrate() (dns/integrate.cpp:138-200), issued on the
// context stream; throws std::runtime_error (with an STX_* code, see
// dns_error_code) on failure.
void dns_advance_one(stx_dns* d);

// Form of the nonlinear terms the next step uses: 0 skew-symmetric, 1
// convective, 2 conservative, -1 Stokes (none).
int dns_next_form(const stx_dns* d);

// The device blocks of a full-state checkpoint, in their fixed order.
std::vector<std::pair<double*, size_t>> dns_state_blocks(stx_dns* d);

// Host part of the state (step, time, alternating switch, ...) saved beside
// the blocks, and put back (the BCs of the restored time re-evaluated; a
// captured step graph dropped).
struct DnsHostState {
  int step = 0, toggle = 1, navg = 0;
  double time = 0.0;
  bool sfd_started = false;
};
DnsHostState dns_host_state(const stx_dns* d);
void dns_set_host_state(stx_dns* d, const DnsHostState& s);

// STX_* status of an exception thrown by the functions above.
int dns_error_code(const std::exception& e);

}  // namespace stx
