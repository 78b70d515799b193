// Implementation of the drop-in C++ surface (vanguard_shim.h) over the C ABI of libvanguard_slic.so.
//
// Model classes hold primitives exactly as the reference's do and implement the closed-form conversions callers
// use on the host; everything grid-sized (solve, solve2D, the per-sweep updates, the CFL maximum) runs through the
// C ABI on the GPU.  Defaults of every constructor follow the reference's: Euler/eulermaterialparameters.cpp:3-34,
// Euler/eulerstatevector.cpp:3-34, MHD/mhdmaterialparameters.cpp:3-19, MHD/mhdstatevector.cpp:3-33,
// HPR/hprmaterialparameters.cpp:3-69, HPR/hprstatevector.cpp:3-33.
#include "vanguard_shim.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <tuple>

#include "../../include/vanguard_slic.h"

namespace {

[[noreturn]] void raise(vg_status st, const char* where) {
    throw std::runtime_error(std::string(where) + ": " + vg_status_string(st) + ": " + vg_last_error_string());
}

void check(vg_status st, const char* where) {
    if (st != VG_OK) raise(st, where);
}

int device() {
    const char* d = std::getenv("VG_DEVICE");
    return d ? std::atoi(d) : 0;
}

int precision() {
    const char* p = std::getenv("VG_PRECISION");
    return (p && std::strcmp(p, "mixed") == 0) ? VG_MIXED : VG_FP64;
}

struct SolverDeleter {
    void operator()(vg_solver* s) const { vg_destroy(s); }
};
using SolverPtr = std::unique_ptr<vg_solver, SolverDeleter>;

// prec < 0: the form VG_PRECISION selects
SolverPtr make_solver(int model, int nx, int ny, int boundary, const double* params, int nparams, int prec = -1) {
    vg_grid_desc d{};
    d.model = model;
    d.nx = nx;
    d.ny = ny;
    d.precision = prec < 0 ? precision() : prec;
    d.boundary = boundary;
    d.device = device();
    for (int i = 0; i < nparams && i < VG_MAX_PARAMS; i++) d.params[i] = params[i];
    vg_solver* s = nullptr;
    check(vg_create(&d, &s), "vg_create");
    return SolverPtr(s);
}

// One cached solver per thread for the per-sweep entry points (a sweep per call would otherwise reallocate).
vg_solver* cached_solver(int model, int nx, int ny, int boundary, const double* params, int nparams) {
    thread_local std::map<std::tuple<int, int, int, int, int, std::string>, SolverPtr> cache;
    std::string key(reinterpret_cast<const char*>(params), sizeof(double) * nparams);
    auto k = std::make_tuple(model, nx, ny, boundary, precision(), key);
    auto it = cache.find(k);
    if (it == cache.end()) it = cache.emplace(k, make_solver(model, nx, ny, boundary, params, nparams)).first;
    return it->second.get();
}

// Runs solve()/solve2D()'s time loop (finalTime-driven) on reference-order primitive planes, in place.
// maxSteps > 0 also stops the loop after that many steps (the shim's step-count overloads).
void run_planes(int model, std::vector<double>& planes, int nx, int ny, const double* params, int nparams, double dx,
                double cfl, double tEnd, double bias, int limiter, int subcycles, int maxSteps = 0, int order = 2,
                int reinit = 0) {
    // the first-order loop runs in the exact form, bit for bit with the reference; the Euler multiphysics, MHD and HPR
    // two-material models have no mixed form
    const bool exact = order == 1 || model == VG_MODEL_EULER_MULTIPHYSICS || model == VG_MODEL_MHD_REDUCED ||
                       model == VG_MODEL_MHD_INTERMEDIATE || model == VG_MODEL_HPR_REDUCED ||
                       model == VG_MODEL_HPR_INTERMEDIATE || model == VG_MODEL_HPR_MULTIPHYSICS ||
                       model == VG_MODEL_MHD_MULTIPHYSICS;
    SolverPtr s = make_solver(model, nx, ny, VG_TRANSMISSIVE, params, nparams, exact ? VG_FP64 : -1);
    vg_run_config c{};
    c.dx = dx;
    c.cfl = cfl;
    c.t_end = tEnd;
    c.max_steps = maxSteps;
    c.bias = bias;
    c.limiter = limiter;
    c.subcycles = subcycles;
    c.order = order;
    c.reinit_frequency = reinit;
    vg_status st = vg_solve(s.get(), planes.data(), planes.data(), &c, nullptr, nullptr, nullptr);
    if (st != VG_OK && st != VG_ENAN) raise(st, "vg_solve");  // non-finite results are returned, as the reference does
}

// ---- packing between reference-style cells and SoA primitive planes
constexpr int kMaxPlanes = 32;  // the most primitive planes of any model (the HPR multiphysics state)
template <class S, class Get>
std::vector<double> pack(const std::vector<S>& cells, int nvar, Get get) {
    long n = cells.size();
    std::vector<double> p(nvar * n);
    for (long i = 0; i < n; i++) {
        double w[kMaxPlanes];
        get(cells[i], w);
        for (int v = 0; v < nvar; v++) p[v * n + i] = w[v];
    }
    return p;
}
// Every 2D entry point packs through here.  The reference's 2D ghost insertion reads rows 0 and 1 and columns 0 and 1
// of the grid (Solvers/solvers.cpp:111-130), so a grid with fewer than 2 rows or columns is outside what its solve2D
// and per-sweep functions define; the device would otherwise treat a single row as a 1D grid.
template <class S>
void require_2d(const std::vector<std::vector<S> >& cells) {
    if (cells.size() < 2 || cells[0].size() < 2)
        throw std::invalid_argument("2D solver: the grid needs at least 2 rows and 2 columns (use the 1D solve for a "
                                    "single row)");
}
template <class S, class Get>
std::vector<double> pack2(const std::vector<std::vector<S> >& cells, int nvar, Get get) {
    require_2d(cells);
    long ny = cells.size(), nx = cells[0].size(), n = nx * ny;
    std::vector<double> p(nvar * n);
    for (long i = 0; i < ny; i++)
        for (long j = 0; j < nx; j++) {
            double w[kMaxPlanes];
            get(cells[i][j], w);
            for (int v = 0; v < nvar; v++) p[v * n + i * nx + j] = w[v];
        }
    return p;
}

void euler_get(const EulerStateVector& c, double* w) {
    w[0] = c.getDensity(), w[1] = c.getXVelocity(), w[2] = c.getYVelocity(), w[3] = c.getZVelocity();
    w[4] = c.getPressure(), w[5] = c.getReactionProgress();
}
EulerStateVector euler_make(const double* w) { return EulerStateVector(w[0], w[1], w[2], w[3], w[4], w[5]); }
void mhd_get(const MHDStateVector& c, double* w) {
    std::vector<double> v = c.computePrimitiveVariableVector();
    for (int i = 0; i < 9; i++) w[i] = v[i];
}
MHDStateVector mhd_make(const double* w) { return MHDStateVector(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], w[8]); }
void hpr_get(const HPRStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 17); }
void reduced_get(const EulerReducedStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 7); }
EulerReducedStateVector reduced_make(const double* w) {
    EulerReducedStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 7);
    return s;
}

HPRStateVector hpr_make(const double* w) {
    HPRStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 17);
    return s;
}

template <class S, class Make>
std::vector<S> unpack(const std::vector<double>& p, long n, int nvar, Make make) {
    std::vector<S> out;
    out.reserve(n);
    for (long i = 0; i < n; i++) {
        double w[kMaxPlanes];
        for (int v = 0; v < nvar; v++) w[v] = p[v * n + i];
        out.push_back(make(w));
    }
    return out;
}
template <class S, class Make>
std::vector<std::vector<S> > unpack2(const std::vector<double>& p, long nx, long ny, int nvar, Make make) {
    std::vector<std::vector<S> > out(ny);
    long n = nx * ny;
    for (long i = 0; i < ny; i++) {
        out[i].reserve(nx);
        for (long j = 0; j < nx; j++) {
            double w[kMaxPlanes];
            for (int v = 0; v < nvar; v++) w[v] = p[v * n + i * nx + j];
            out[i].push_back(make(w));
        }
    }
    return out;
}

void euler_params(const EulerMaterialParameters& mp, double* prm) {
    prm[0] = mp.getAdiabaticIndex(), prm[1] = mp.getStiffeningParameter(), prm[2] = mp.getSpecificHeatCapacity();
    prm[3] = mp.getEnergyOfFormation(), prm[4] = mp.getIgnitionTemperature(), prm[5] = mp.getReactionRate();
}
void mhd_params(const MHDMaterialParameters& mp, double* prm) {
    prm[0] = mp.getAdiabaticIndex(), prm[1] = mp.getStiffeningParameter(), prm[2] = mp.getHyperbolicWaveSpeed();
}
void hpr_params(const HPRMaterialParameters& mp, double* prm) {
    const string& eos = mp.getEquationOfState();
    if (eos != "StiffenedGas" && eos != "ShockMieGruneisen" && eos != "GodunovRomenski")
        throw std::runtime_error("HPR: unknown equation of state '" + eos + "'");
    prm[12] = eos == "StiffenedGas" ? 0.0 : eos == "ShockMieGruneisen" ? 1.0 : 2.0;
    prm[13] = mp.getReferenceGruneisenCoefficient(), prm[14] = mp.getReferenceSoundSpeed();
    prm[15] = mp.getHugoniotSlopeCoefficient(), prm[16] = mp.getAlphaParameter();
    prm[17] = mp.getIsPlastic() ? 1.0 : 0.0, prm[18] = mp.getElasticPlasticTransitionParameter();
    prm[19] = mp.getPowerLawIndex();
    prm[0] = mp.getAdiabaticIndex(), prm[1] = mp.getStiffeningParameter(), prm[2] = mp.getSpecificHeatCapacity();
    prm[3] = mp.getReferenceDensity(), prm[4] = mp.getInitialTemperature(), prm[5] = mp.getTransverseWaveSpeed();
    prm[6] = mp.getHeatWaveSpeed(), prm[7] = mp.getStrainDissipationTime(), prm[8] = mp.getThermalImpulseRelaxationTime();
    prm[9] = mp.getReferenceTemperature(), prm[10] = mp.getReferencePressure(), prm[11] = mp.getIsThermal() ? 1.0 : 0.0;
}

// Boundary kind of a caller-built ghosted array along one line: the reference's transmissive mirror
// (Solvers/solvers.cpp:17-23) or wrap-around; anything else cannot be expressed by the GPU path.
template <class Eq>
int boundary_kind(long n, Eq same) {
    // same(g, c): ghost slot g (0..n+3) holds interior cell c
    if (same(0, 1) && same(1, 0) && same(n + 2, n - 1) && same(n + 3, n - 2)) return VG_TRANSMISSIVE;
    if (same(0, n - 2) && same(1, n - 1) && same(n + 2, 0) && same(n + 3, 1)) return VG_PERIODIC;
    return -1;
}

template <class S, class Get>
bool equal_cells(const S& a, const S& b, int nvar, Get get) {
    double wa[kMaxPlanes], wb[kMaxPlanes];
    get(a, wa);
    get(b, wb);
    return std::memcmp(wa, wb, sizeof(double) * nvar) == 0;
}

template <class S, class Get, class Make>
void sweep2d(int model, int nvar, std::vector<std::vector<S> >& cells, std::vector<std::vector<S> >& withB, int axis,
             double dx, double dt, double bias, int limiter, const double* prm, int nprm, Get get, Make make) {
    long ny = cells.size(), nx = cells[0].size();
    if ((long)withB.size() != ny + 4 || (long)withB[0].size() != nx + 4)
        throw std::runtime_error("sweep: the ghosted array must have 2 ghost cells on every side");
    int bc = -1;
    for (long line = 0; line < (axis == 0 ? ny : nx); line++) {
        int k = axis == 0 ? boundary_kind(nx, [&](long g, long c) { return equal_cells(withB[line + 2][g], cells[line][c], nvar, get); })
                          : boundary_kind(ny, [&](long g, long c) { return equal_cells(withB[g][line + 2], cells[c][line], nvar, get); });
        if (k < 0 || (bc >= 0 && k != bc))
            throw std::runtime_error("sweep: ghost cells other than transmissive or periodic copies are not supported");
        bc = k;
    }
    vg_solver* s = cached_solver(model, (int)nx, (int)ny, bc, prm, nprm);
    std::vector<double> planes = pack2(cells, nvar, get);
    check(vg_upload_primitive(s, planes.data(), 0, nullptr), "vg_upload_primitive");
    check(vg_sweep(s, axis, dx, dt, bias, limiter, nullptr), "vg_sweep");
    check(vg_download_primitive(s, planes.data(), 0, nullptr), "vg_download_primitive");
    cells = unpack2<S>(planes, nx, ny, nvar, make);
}

}  // namespace

// ------------------------------------------------------------------------------------------- Euler model
EulerMaterialParameters::EulerMaterialParameters() : EulerMaterialParameters(1.0, 0.0) {}
EulerMaterialParameters::EulerMaterialParameters(double g) : EulerMaterialParameters(g, 0.0) {}
EulerMaterialParameters::EulerMaterialParameters(double g, double pinf) : EulerMaterialParameters(g, pinf, 25.0, 0.0, 0.25, 250.0) {}
EulerMaterialParameters::EulerMaterialParameters(double g, double pinf, double cv, double e0, double tign, double rate)
    : adiabaticIndex(g), stiffeningParameter(pinf), specificHeatCapacity(cv), energyOfFormation(e0), ignitionTemperature(tign),
      reactionRate(rate) {}

double EulerEquationOfState::computeSpecificInternalEnergy(double rho, double p, EulerMaterialParameters mp) {
    double g = mp.getAdiabaticIndex();
    return (p + (g * mp.getStiffeningParameter())) / ((g - 1) * rho);
}
double EulerEquationOfState::computePressure(double rho, double e, EulerMaterialParameters mp) {
    double g = mp.getAdiabaticIndex();
    return ((e * (g - 1)) * rho) - (g * mp.getStiffeningParameter());
}
double EulerEquationOfState::computeSoundSpeed(double rho, double p, EulerMaterialParameters mp) {
    return std::sqrt((mp.getAdiabaticIndex() * (p + mp.getStiffeningParameter())) / rho);
}

EulerStateVector::EulerStateVector() : EulerStateVector(1.0, 0.0, 0.0, 0.0, 1.0, 1.0) {}
EulerStateVector::EulerStateVector(double r, double u, double v, double w, double p) : EulerStateVector(r, u, v, w, p, 1.0) {}
EulerStateVector::EulerStateVector(double r, double u, double v, double w, double p, double lam)
    : density(r), xVelocity(u), yVelocity(v), zVelocity(w), pressure(p), reactionProgress(lam) {}

void EulerStateVector::setPrimitiveVariableVector(vector<double> w) {
    density = w[0], xVelocity = w[1], yVelocity = w[2], zVelocity = w[3], pressure = w[4], reactionProgress = w[5];
}
vector<double> EulerStateVector::computePrimitiveVariableVector() const {
    return {density, xVelocity, yVelocity, zVelocity, pressure, reactionProgress};
}
double EulerStateVector::computeSpecificInternalEnergy(EulerMaterialParameters mp) const {
    return EulerEquationOfState::computeSpecificInternalEnergy(density, pressure, mp);
}
double EulerStateVector::computeTotalEnergy(EulerMaterialParameters mp) const {
    double v2 = ((xVelocity * xVelocity) + (yVelocity * yVelocity)) + (zVelocity * zVelocity);
    return density * (((0.5 * v2) + computeSpecificInternalEnergy(mp)) + (mp.getEnergyOfFormation() * (reactionProgress - 1.0)));
}
double EulerStateVector::computeSoundSpeed(EulerMaterialParameters mp) const {
    return EulerEquationOfState::computeSoundSpeed(density, pressure, mp);
}
vector<double> EulerStateVector::computeConservedVariableVector(EulerMaterialParameters mp) const {
    return {density, density * xVelocity, density * yVelocity, density * zVelocity, computeTotalEnergy(mp), density * reactionProgress};
}
void EulerStateVector::setConservedVariableVector(vector<double> u, EulerMaterialParameters mp) {
    density = u[0];
    xVelocity = u[1] / density, yVelocity = u[2] / density, zVelocity = u[3] / density;
    reactionProgress = u[5] / density;
    double v2 = ((xVelocity * xVelocity) + (yVelocity * yVelocity)) + (zVelocity * zVelocity);
    double e = ((u[4] / density) - (0.5 * v2)) - (mp.getEnergyOfFormation() * (reactionProgress - 1.0));
    pressure = EulerEquationOfState::computePressure(density, e, mp);
}
static vector<double> euler_flux(const vector<double>& u, EulerMaterialParameters mp, int axis) {
    double rho = u[0], vx = u[1] / rho, vy = u[2] / rho, vz = u[3] / rho, lam = u[5] / rho;
    double v2 = ((vx * vx) + (vy * vy)) + (vz * vz);
    double E = u[4] / rho;
    double p = EulerEquationOfState::computePressure(rho, (E - (0.5 * v2)) - (mp.getEnergyOfFormation() * (lam - 1.0)), mp);
    double un = axis == 0 ? vx : vy;
    vector<double> f = {rho * un, rho * (un * vx), rho * (un * vy), rho * (un * vz), (rho * (un * E)) + (un * p), rho * (un * lam)};
    f[1 + axis] += p;
    return f;
}
vector<double> EulerStateVector::computeXFluxVector(vector<double> u, EulerMaterialParameters mp) { return euler_flux(u, mp, 0); }
vector<double> EulerStateVector::computeYFluxVector(vector<double> u, EulerMaterialParameters mp) { return euler_flux(u, mp, 1); }
vector<double> EulerStateVector::computeXFluxVector(EulerMaterialParameters mp) const {
    return computeXFluxVector(computeConservedVariableVector(mp), mp);
}
vector<double> EulerStateVector::computeYFluxVector(EulerMaterialParameters mp) const {
    return computeYFluxVector(computeConservedVariableVector(mp), mp);
}

// --------------------------------------------------------------------------------------------- MHD model
MHDMaterialParameters::MHDMaterialParameters() : adiabaticIndex(1.0), stiffeningParameter(0.0), hyperbolicWaveSpeed(2.0),
                                                 parabolicDamping(std::sqrt(0.36)) {}
MHDMaterialParameters::MHDMaterialParameters(double g) : adiabaticIndex(g), stiffeningParameter(0.0), hyperbolicWaveSpeed(0.0),
                                                         parabolicDamping(0.0) {}
void MHDMaterialParameters::configureParabolicDamping() { parabolicDamping = std::sqrt(hyperbolicWaveSpeed * 0.18); }

MHDStateVector::MHDStateVector() : MHDStateVector(1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0) {}
MHDStateVector::MHDStateVector(double r, double u, double v, double w, double p, double bx, double by, double bz, double psi)
    : w_{r, u, v, w, p, bx, by, bz, psi} {}
void MHDStateVector::setPrimitiveVariableVector(vector<double> w) {
    for (int i = 0; i < 9; i++) w_[i] = w[i];
}
vector<double> MHDStateVector::computePrimitiveVariableVector() const { return vector<double>(w_, w_ + 9); }
vector<double> MHDStateVector::computeConservedVariableVector(MHDMaterialParameters mp) const {
    double r = w_[0], u = w_[1], v = w_[2], w = w_[3], p = w_[4], g = mp.getAdiabaticIndex();
    double e = (p + (g * mp.getStiffeningParameter())) / ((g - 1) * r);
    double hydro = r * ((0.5 * (((u * u) + (v * v)) + (w * w))) + e);
    double b2 = ((w_[5] * w_[5]) + (w_[6] * w_[6])) + (w_[7] * w_[7]);
    return {r, r * u, r * v, r * w, hydro + (0.5 * b2), w_[5], w_[6], w_[7], w_[8]};
}
void MHDStateVector::setConservedVariableVector(vector<double> U, MHDMaterialParameters mp) {
    double r = U[0], g = mp.getAdiabaticIndex();
    double u = U[1] / r, v = U[2] / r, w = U[3] / r;
    double b2 = ((U[5] * U[5]) + (U[6] * U[6])) + (U[7] * U[7]);
    double e = ((U[4] - (0.5 * b2)) / r) - (0.5 * (((u * u) + (v * v)) + (w * w)));
    double p = ((e * (g - 1)) * r) - (g * mp.getStiffeningParameter());
    double nw[9] = {r, u, v, w, p, U[5], U[6], U[7], U[8]};
    std::memcpy(w_, nw, sizeof(nw));
}

// --------------------------------------------------------------------------------------------- HPR model
HPRMaterialParameters::HPRMaterialParameters()
    : HPRMaterialParameters("StiffenedGas", false, false, 8.31445985, 1.0, 1.0 / 1.4, 0.0, 0.0, 1.0, 1.4, 0.0, 0.0, 0.0, 0.0,
                            0.0, 1.0, 0.0, 0.0, std::pow(10.0, -2.0), 0.75, 0.0, 1.0, std::pow(10.0, -16.0), 0.0, 0.0, 0.0) {}
HPRMaterialParameters::HPRMaterialParameters(string eos, bool thermal, bool plastic, double R, double rho0, double pref,
                                             double tref, double t0, double cv, double g, double pinf, double c0, double gr0,
                                             double s, double e0, double cs, double tau1, double tau2, double mu, double pr,
                                             double sy, double n, double alpha, double a, double b, double c)
    : equationOfState(eos), isThermal(thermal), isPlastic(plastic), idealGasConstant(R), referenceDensity(rho0),
      referencePressure(pref), referenceTemperature(tref), initialTemperature(t0), specificHeatCapacity(cv), adiabaticIndex(g),
      stiffeningParameter(pinf), referenceSoundSpeed(c0), referenceGruneisenCoefficient(gr0), hugoniotSlopeCoefficient(s),
      referenceInternalEnergy(e0), transverseWaveSpeed(cs), strainDissipationTime(tau1), thermalImpulseRelaxationTime(tau2),
      dynamicViscosityCoefficient(mu), prandtlNumber(pr), elasticPlasticTransitionParameter(sy), powerLawIndex(n),
      heatWaveSpeed(alpha), alphaParameter(a), betaParameter(b), gammaParameter(c) {}
// HPR/hprmaterialparameters.cpp:71-119
double HPRMaterialParameters::computeStrainDissipationTime() const {
    return 6.0 * (dynamicViscosityCoefficient / (referencePressure * (transverseWaveSpeed * transverseWaveSpeed)));
}
double HPRMaterialParameters::computeHeatConductionCoefficient() const {
    return dynamicViscosityCoefficient * adiabaticIndex * (specificHeatCapacity / prandtlNumber);
}
double HPRMaterialParameters::computeThermalImpulseRelaxationTime(double kappa) const {
    return kappa * (referenceDensity / (initialTemperature * (heatWaveSpeed * heatWaveSpeed)));
}
double HPRMaterialParameters::computeThermalImpulseRelaxationTime() const {
    return computeThermalImpulseRelaxationTime(computeHeatConductionCoefficient());
}
void HPRMaterialParameters::configureStrainDissipationTime() { strainDissipationTime = computeStrainDissipationTime(); }
void HPRMaterialParameters::configureThermalImpulseRelaxationTime() {
    thermalImpulseRelaxationTime = computeThermalImpulseRelaxationTime();
}
void HPRMaterialParameters::configureThermalImpulseRelaxationTime(double kappa) {
    thermalImpulseRelaxationTime = computeThermalImpulseRelaxationTime(kappa);
}

HPRStateVector::HPRStateVector() {
    std::memset(w_, 0, sizeof(w_));
    double c = std::pow(1.0, 1.0 / 3.0);
    w_[0] = 1.0;
    w_[1] = 1.0 / 1.4;
    w_[2] = w_[6] = w_[10] = c;
}
HPRStateVector::HPRStateVector(double rho, double p, vector<vector<double> > A, double u, double v, double w, double jx,
                               double jy, double jz) {
    w_[0] = rho, w_[1] = p;
    setDistortionTensor(A);
    w_[11] = u, w_[12] = v, w_[13] = w, w_[14] = jx, w_[15] = jy, w_[16] = jz;
}
vector<vector<double> > HPRStateVector::getDistortionTensor() const {
    vector<vector<double> > A(3, vector<double>(3));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = w_[2 + 3 * i + j];
    return A;
}
void HPRStateVector::setDistortionTensor(vector<vector<double> > A) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) w_[2 + 3 * i + j] = A[i][j];
}

// ----------------------------------------------------------------------------------------- slope limiters
double SlopeLimiters::computeRCoefficient(double r, double w) { return 2.0 / ((1.0 - w) + ((1.0 + w) * r)); }
double SlopeLimiters::computeSuperBeeSlopeLimiter(double r, double w) {
    if (r < 0.0) return 0.0;
    if (r < 0.5) return 2.0 * r;
    if (r < 1.0) return 1.0;
    double xi = computeRCoefficient(r, w), m = (xi < r) ? xi : r;
    return (2.0 < m) ? 2.0 : m;
}
double SlopeLimiters::computeVanLeerSlopeLimiter(double r, double w) {
    if (r < 0.0) return 0.0;
    double a = (2.0 * r) / (1.0 + r), b = computeRCoefficient(r, w);
    return (b < a) ? b : a;
}
double SlopeLimiters::computeMinBeeSlopeLimiter(double r, double w) {
    if (r < 0.0) return 0.0;
    if (r < 1.0) return r;
    double b = computeRCoefficient(r, w);
    return (b < 1.0) ? b : 1.0;
}
double SlopeLimiters::computeSlopeLimiter(double r, double w, int id) {
    return id == 0 ? computeSuperBeeSlopeLimiter(r, w) : id == 1 ? computeVanLeerSlopeLimiter(r, w) : computeMinBeeSlopeLimiter(r, w);
}

// ------------------------------------------------------------------------------------------ solver helpers
vector<EulerStateVector> Solvers::insertBoundaryCells(vector<EulerStateVector>& c, int b) {
    long n = c.size();
    vector<EulerStateVector> g(n + 2 * b);
    for (long i = 0; i < n; i++) g[i + b] = c[i];
    for (int k = 0; k < b; k++) {
        g[b - 1 - k] = c[k < n ? k : n - 1];
        g[n + b + k] = c[n - 1 - k >= 0 ? n - 1 - k : 0];
    }
    return g;
}
vector<vector<EulerStateVector> > Solvers::insertBoundaryCells2D(vector<vector<EulerStateVector> >& c, int b) {
    long ny = c.size(), nx = c[0].size();
    vector<vector<EulerStateVector> > g(ny + 2 * b, vector<EulerStateVector>(nx + 2 * b));
    for (long i = 0; i < ny; i++)
        for (long j = 0; j < nx; j++) g[i + b][j + b] = c[i][j];
    for (long i = 0; i < ny; i++)
        for (int k = 0; k < b; k++) {
            g[i + b][b - 1 - k] = c[i][k];
            g[i + b][nx + b + k] = c[i][nx - 1 - k];
        }
    for (long j = 0; j < nx; j++)
        for (int k = 0; k < b; k++) {
            g[b - 1 - k][j + b] = c[k][j];
            g[ny + b + k][j + b] = c[ny - 1 - k][j];
        }
    return g;  // corner blocks keep the default state, as the reference's do
}
double Solvers::computeMaximumWaveSpeed(vector<EulerStateVector>& cells, EulerMaterialParameters mp) {
    double prm[6];
    euler_params(mp, prm);
    std::vector<double> p = pack(cells, 6, euler_get);
    vg_solver* s = cached_solver(VG_MODEL_EULER, (int)cells.size(), 1, VG_TRANSMISSIVE, prm, 6);
    check(vg_upload_primitive(s, p.data(), 0, nullptr), "vg_upload_primitive");
    double out = 0.0;
    check(vg_max_wave_speed(s, &out, nullptr), "vg_max_wave_speed");
    return out;
}
double Solvers::computeMaximumWaveSpeed2D(vector<vector<EulerStateVector> >& cells, EulerMaterialParameters mp) {
    // the maximum over exactly the cells given, as the reference helper takes it: a ghosted array brings its own
    // default-constructed corners, an interior-only array has none
    double prm[6];
    euler_params(mp, prm);
    std::vector<double> p = pack2(cells, 6, euler_get);
    vg_solver* s = cached_solver(VG_MODEL_EULER, (int)cells[0].size(), (int)cells.size(), VG_TRANSMISSIVE, prm, 6);
    check(vg_upload_primitive(s, p.data(), 0, nullptr), "vg_upload_primitive");
    double out = 0.0;
    check(vg_max_wave_speed_cells(s, &out, nullptr), "vg_max_wave_speed_cells");
    return out;
}
double Solvers::computeStableTimeStep(double dt, double t, double tEnd, int it) {
    double d = dt;
    if (it <= 5) d *= 0.2;
    if ((t + d) > tEnd) d = tEnd - t;
    return d;
}
double Solvers::computeStableTimeStep(vector<EulerStateVector>& cells, double dx, double cfl, double t, double tEnd, int it,
                                      EulerMaterialParameters mp) {
    return computeStableTimeStep(cfl * (dx / computeMaximumWaveSpeed(cells, mp)), t, tEnd, it);
}
double Solvers::computeStableTimeStep2D(vector<vector<EulerStateVector> >& cells, double dx, double cfl, double t, double tEnd,
                                        int it, EulerMaterialParameters mp) {
    return computeStableTimeStep(cfl * (dx / computeMaximumWaveSpeed2D(cells, mp)), t, tEnd, it);
}

// ------------------------------------------------------------------------------------------- Euler solver
void SecondOrderSolver::computeSLICTimeStep(vector<EulerStateVector>& cells, vector<EulerStateVector>& withB, double dx,
                                            double dt, double bias, int limiter, EulerMaterialParameters mp) {
    long n = cells.size();
    if ((long)withB.size() != n + 4) throw std::runtime_error("computeSLICTimeStep: need 2 ghost cells per side");
    int bc = boundary_kind(n, [&](long g, long c) { return equal_cells(withB[g], cells[c], 6, euler_get); });
    if (bc < 0) throw std::runtime_error("computeSLICTimeStep: ghost cells other than transmissive or periodic copies");
    double prm[6];
    euler_params(mp, prm);
    vg_solver* s = cached_solver(VG_MODEL_EULER, (int)n, 1, bc, prm, 6);
    std::vector<double> p = pack(cells, 6, euler_get);
    check(vg_upload_primitive(s, p.data(), 0, nullptr), "vg_upload_primitive");
    check(vg_sweep(s, 0, dx, dt, bias, limiter, nullptr), "vg_sweep");
    check(vg_download_primitive(s, p.data(), 0, nullptr), "vg_download_primitive");
    cells = unpack<EulerStateVector>(p, n, 6, euler_make);
}
void SecondOrderSolver::computeXSLICTimeStep2D(vector<vector<EulerStateVector> >& cells, vector<vector<EulerStateVector> >& withB,
                                               double dx, double dt, double bias, int limiter, EulerMaterialParameters mp) {
    double prm[6];
    euler_params(mp, prm);
    sweep2d(VG_MODEL_EULER, 6, cells, withB, 0, dx, dt, bias, limiter, prm, 6, euler_get, euler_make);
}
void SecondOrderSolver::computeYSLICTimeStep2D(vector<vector<EulerStateVector> >& cells, vector<vector<EulerStateVector> >& withB,
                                               double dx, double dt, double bias, int limiter, EulerMaterialParameters mp) {
    double prm[6];
    euler_params(mp, prm);
    sweep2d(VG_MODEL_EULER, 6, cells, withB, 1, dx, dt, bias, limiter, prm, 6, euler_get, euler_make);
}
vector<EulerStateVector> SecondOrderSolver::solve(vector<EulerStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                  double bias, int limiter, int subcycles, EulerMaterialParameters mp) {
    return solve(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, mp, 0);
}
vector<EulerStateVector> SecondOrderSolver::solve(vector<EulerStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                  double bias, int limiter, int /*subcycles: no source in the Euler model*/,
                                                  EulerMaterialParameters mp, int maxSteps) {
    double prm[6];
    euler_params(mp, prm);
    std::vector<double> p = pack(initialCells, 6, euler_get);
    run_planes(VG_MODEL_EULER, p, (int)initialCells.size(), 1, prm, 6, dx, cfl, tEnd, bias, limiter, 0, maxSteps);
    return unpack<EulerStateVector>(p, initialCells.size(), 6, euler_make);
}
vector<vector<EulerStateVector> > SecondOrderSolver::solve2D(vector<vector<EulerStateVector> >& initialCells, double dx,
                                                             double cfl, double tEnd, double bias, int limiter, int subcycles,
                                                             EulerMaterialParameters mp) {
    return solve2D(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, mp, 0);
}
vector<vector<EulerStateVector> > SecondOrderSolver::solve2D(vector<vector<EulerStateVector> >& initialCells, double dx,
                                                             double cfl, double tEnd, double bias, int limiter, int,
                                                             EulerMaterialParameters mp, int maxSteps) {
    double prm[6];
    euler_params(mp, prm);
    std::vector<double> p = pack2(initialCells, 6, euler_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_EULER, p, (int)nx, (int)ny, prm, 6, dx, cfl, tEnd, bias, limiter, 0, maxSteps);
    return unpack2<EulerStateVector>(p, nx, ny, 6, euler_make);
}

// ----------------------------------------------------------------------------------- reduced two-material
EulerReducedStateVector::EulerReducedStateVector() : EulerReducedStateVector(0.999, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0) {}
EulerReducedStateVector::EulerReducedStateVector(double a1, double u, double v, double w, double r1, double r2, double p)
    : w_{a1, u, v, w, r1, r2, p} {}
void EulerReducedStateVector::setPrimitiveVariableVector(vector<double> w) {
    for (int i = 0; i < 7; i++) w_[i] = w[i];
}
vector<double> EulerReducedStateVector::computePrimitiveVariableVector() const { return vector<double>(w_, w_ + 7); }

EulerMultiphysicsStateVector::EulerMultiphysicsStateVector()
    : EulerMultiphysicsStateVector(0.999, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0) {}
EulerMultiphysicsStateVector::EulerMultiphysicsStateVector(double a1, double u, double v, double w, double r1, double p1,
                                                           double r2, double p2)
    : w_{a1, u, v, w, r1, p1, r2, p2} {}
void EulerMultiphysicsStateVector::setPrimitiveVariableVector(vector<double> w) {
    for (int i = 0; i < 8; i++) w_[i] = w[i];
}
vector<double> EulerMultiphysicsStateVector::computePrimitiveVariableVector() const { return vector<double>(w_, w_ + 8); }

namespace {
void mph_get(const EulerMultiphysicsStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 8); }
EulerMultiphysicsStateVector mph_make(const double* w) {
    EulerMultiphysicsStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 8);
    return s;
}
void reduced_params(const EulerMaterialParameters& m1, const EulerMaterialParameters& m2, double* prm) {
    prm[0] = m1.getAdiabaticIndex(), prm[1] = m1.getStiffeningParameter();
    prm[2] = m2.getAdiabaticIndex(), prm[3] = m2.getStiffeningParameter();
}
}  // namespace

vector<EulerReducedStateVector> SecondOrderSolver::solve(vector<EulerReducedStateVector>& initialCells, double dx, double cfl,
                                                         double tEnd, double bias, int limiter, int subcycles, int reinit,
                                                         EulerMaterialParameters m1, EulerMaterialParameters m2) {
    return solve(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, reinit, m1, m2, 0);
}
vector<EulerReducedStateVector> SecondOrderSolver::solve(vector<EulerReducedStateVector>& initialCells, double dx, double cfl,
                                                         double tEnd, double bias, int limiter,
                                                         int /*subcycles: the reference's loop body is empty*/, int reinit,
                                                         EulerMaterialParameters m1, EulerMaterialParameters m2,
                                                         int maxSteps) {
    double prm[4];
    reduced_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 7, reduced_get);
    run_planes(VG_MODEL_EULER_REDUCED, p, (int)initialCells.size(), 1, prm, 4, dx, cfl, tEnd, bias, limiter, 0, maxSteps,
               2, reinit);
    return unpack<EulerReducedStateVector>(p, initialCells.size(), 7, reduced_make);
}
vector<vector<EulerReducedStateVector> > SecondOrderSolver::solve2D(vector<vector<EulerReducedStateVector> >& initialCells,
                                                                    double dx, double cfl, double tEnd, double bias,
                                                                    int limiter, int subcycles, int reinit,
                                                                    EulerMaterialParameters m1, EulerMaterialParameters m2) {
    return solve2D(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, reinit, m1, m2, 0);
}
vector<vector<EulerReducedStateVector> > SecondOrderSolver::solve2D(vector<vector<EulerReducedStateVector> >& initialCells,
                                                                    double dx, double cfl, double tEnd, double bias,
                                                                    int limiter, int, int reinit, EulerMaterialParameters m1,
                                                                    EulerMaterialParameters m2, int maxSteps) {
    double prm[4];
    reduced_params(m1, m2, prm);
    std::vector<double> p = pack2(initialCells, 7, reduced_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_EULER_REDUCED, p, (int)nx, (int)ny, prm, 4, dx, cfl, tEnd, bias, limiter, 0, maxSteps, 2, reinit);
    return unpack2<EulerReducedStateVector>(p, nx, ny, 7, reduced_make);
}

vector<EulerMultiphysicsStateVector> SecondOrderSolver::solve(vector<EulerMultiphysicsStateVector>& initialCells, double dx,
                                                              double cfl, double tEnd, double bias, int limiter, int,
                                                              int reinit, EulerMaterialParameters m1,
                                                              EulerMaterialParameters m2) {
    double prm[4];
    reduced_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 8, mph_get);
    run_planes(VG_MODEL_EULER_MULTIPHYSICS, p, (int)initialCells.size(), 1, prm, 4, dx, cfl, tEnd, bias, limiter, 0, 0, 2,
               reinit);
    return unpack<EulerMultiphysicsStateVector>(p, initialCells.size(), 8, mph_make);
}
vector<vector<EulerMultiphysicsStateVector> > SecondOrderSolver::solve2D(
    vector<vector<EulerMultiphysicsStateVector> >& initialCells, double dx, double cfl, double tEnd, double bias,
    int limiter, int, int reinit, EulerMaterialParameters m1, EulerMaterialParameters m2) {
    double prm[4];
    reduced_params(m1, m2, prm);
    std::vector<double> p = pack2(initialCells, 8, mph_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_EULER_MULTIPHYSICS, p, (int)nx, (int)ny, prm, 4, dx, cfl, tEnd, bias, limiter, 0, 0, 2, reinit);
    return unpack2<EulerMultiphysicsStateVector>(p, nx, ny, 8, mph_make);
}

// --------------------------------------------------------------------------------------------- MHD solver
void MHDSecondOrderSolver::computeXSLICTimeStep2D(vector<vector<MHDStateVector> >& cells, vector<vector<MHDStateVector> >& withB,
                                                  double dx, double dt, double bias, int limiter, MHDMaterialParameters mp) {
    double prm[3];
    mhd_params(mp, prm);
    sweep2d(VG_MODEL_MHD, 9, cells, withB, 0, dx, dt, bias, limiter, prm, 3, mhd_get, mhd_make);
}
void MHDSecondOrderSolver::computeYSLICTimeStep2D(vector<vector<MHDStateVector> >& cells, vector<vector<MHDStateVector> >& withB,
                                                  double dx, double dt, double bias, int limiter, MHDMaterialParameters mp) {
    double prm[3];
    mhd_params(mp, prm);
    sweep2d(VG_MODEL_MHD, 9, cells, withB, 1, dx, dt, bias, limiter, prm, 3, mhd_get, mhd_make);
}
vector<MHDStateVector> MHDSecondOrderSolver::solve(vector<MHDStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                   double bias, int limiter, int subcycles, MHDMaterialParameters mp) {
    return solve(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, mp, 0);
}
vector<MHDStateVector> MHDSecondOrderSolver::solve(vector<MHDStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                   double bias, int limiter, int subcycles, MHDMaterialParameters mp,
                                                   int maxSteps) {
    double prm[3];
    mhd_params(mp, prm);
    std::vector<double> p = pack(initialCells, 9, mhd_get);
    run_planes(VG_MODEL_MHD, p, (int)initialCells.size(), 1, prm, 3, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps);
    return unpack<MHDStateVector>(p, initialCells.size(), 9, mhd_make);
}
vector<vector<MHDStateVector> > MHDSecondOrderSolver::solve2D(vector<vector<MHDStateVector> >& initialCells, double dx, double cfl,
                                                              double tEnd, double bias, int limiter, int subcycles,
                                                              MHDMaterialParameters mp) {
    return solve2D(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, mp, 0);
}
vector<vector<MHDStateVector> > MHDSecondOrderSolver::solve2D(vector<vector<MHDStateVector> >& initialCells, double dx, double cfl,
                                                              double tEnd, double bias, int limiter, int subcycles,
                                                              MHDMaterialParameters mp, int maxSteps) {
    double prm[3];
    mhd_params(mp, prm);
    std::vector<double> p = pack2(initialCells, 9, mhd_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_MHD, p, (int)nx, (int)ny, prm, 3, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps);
    return unpack2<MHDStateVector>(p, nx, ny, 9, mhd_make);
}

// ------------------------------------------------------------------------------------- MHD reduced model
MHDReducedStateVector::MHDReducedStateVector()
    : MHDReducedStateVector(0.999, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0) {}
MHDReducedStateVector::MHDReducedStateVector(double a1, double u, double v, double w, double r1, double r2, double p,
                                             double bx, double by, double bz, double psi)
    : w_{a1, u, v, w, r1, r2, p, bx, by, bz, psi} {}
void MHDReducedStateVector::setPrimitiveVariableVector(vector<double> w) {
    for (int i = 0; i < 11; i++) w_[i] = w[i];
}
vector<double> MHDReducedStateVector::computePrimitiveVariableVector() const { return vector<double>(w_, w_ + 11); }

namespace {
void mred_get(const MHDReducedStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 11); }
MHDReducedStateVector mred_make(const double* w) {
    MHDReducedStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 11);
    return s;
}
// {gamma1, p_inf1, gamma2, p_inf2, c_h}: the second-order loop replaces c_h every step, as solve{,2D} does
void mred_params(const MHDMaterialParameters& m1, const MHDMaterialParameters& m2, double* prm) {
    prm[0] = m1.getAdiabaticIndex(), prm[1] = m1.getStiffeningParameter();
    prm[2] = m2.getAdiabaticIndex(), prm[3] = m2.getStiffeningParameter();
    prm[4] = m1.getHyperbolicWaveSpeed();
}
}  // namespace

vector<MHDReducedStateVector> MHDSecondOrderSolver::solve(vector<MHDReducedStateVector>& initialCells, double dx,
                                                          double cfl, double tEnd, double bias, int limiter,
                                                          int subcycles, int reinit, MHDMaterialParameters m1,
                                                          MHDMaterialParameters m2) {
    return solve(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, reinit, m1, m2, 0);
}
vector<MHDReducedStateVector> MHDSecondOrderSolver::solve(vector<MHDReducedStateVector>& initialCells, double dx,
                                                          double cfl, double tEnd, double bias, int limiter,
                                                          int subcycles, int reinit, MHDMaterialParameters m1,
                                                          MHDMaterialParameters m2, int maxSteps) {
    double prm[5];
    mred_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 11, mred_get);
    run_planes(VG_MODEL_MHD_REDUCED, p, (int)initialCells.size(), 1, prm, 5, dx, cfl, tEnd, bias, limiter, subcycles,
               maxSteps, 2, reinit);
    return unpack<MHDReducedStateVector>(p, initialCells.size(), 11, mred_make);
}
vector<vector<MHDReducedStateVector> > MHDSecondOrderSolver::solve2D(vector<vector<MHDReducedStateVector> >& initialCells,
                                                                     double dx, double cfl, double tEnd, double bias,
                                                                     int limiter, int subcycles, int reinit,
                                                                     MHDMaterialParameters m1, MHDMaterialParameters m2) {
    return solve2D(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, reinit, m1, m2, 0);
}
vector<vector<MHDReducedStateVector> > MHDSecondOrderSolver::solve2D(vector<vector<MHDReducedStateVector> >& initialCells,
                                                                     double dx, double cfl, double tEnd, double bias,
                                                                     int limiter, int subcycles, int reinit,
                                                                     MHDMaterialParameters m1, MHDMaterialParameters m2,
                                                                     int maxSteps) {
    double prm[5];
    mred_params(m1, m2, prm);
    std::vector<double> p = pack2(initialCells, 11, mred_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_MHD_REDUCED, p, (int)nx, (int)ny, prm, 5, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps, 2,
               reinit);
    return unpack2<MHDReducedStateVector>(p, nx, ny, 11, mred_make);
}

// -------------------------------------------------------------------------------- MHD intermediate model
MHDIntermediateStateVector::MHDIntermediateStateVector()
    : w_{0.999, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0} {}
void MHDIntermediateStateVector::setPrimitiveVariableVector(vector<double> w) {
    for (int i = 0; i < 12; i++) w_[i] = w[i];
}
vector<double> MHDIntermediateStateVector::computePrimitiveVariableVector() const {
    return vector<double>(w_, w_ + 12);
}

namespace {
void mint_get(const MHDIntermediateStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 12); }
MHDIntermediateStateVector mint_make(const double* w) {
    MHDIntermediateStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 12);
    return s;
}
}  // namespace

vector<MHDIntermediateStateVector> MHDSecondOrderSolver::solve(vector<MHDIntermediateStateVector>& initialCells,
                                                               double dx, double cfl, double tEnd, double bias,
                                                               int limiter, int subcycles, int reinit,
                                                               MHDMaterialParameters m1, MHDMaterialParameters m2) {
    double prm[5];
    mred_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 12, mint_get);
    run_planes(VG_MODEL_MHD_INTERMEDIATE, p, (int)initialCells.size(), 1, prm, 5, dx, cfl, tEnd, bias, limiter,
               subcycles, 0, 2, reinit);
    return unpack<MHDIntermediateStateVector>(p, initialCells.size(), 12, mint_make);
}
vector<vector<MHDIntermediateStateVector> > MHDSecondOrderSolver::solve2D(
    vector<vector<MHDIntermediateStateVector> >& initialCells, double dx, double cfl, double tEnd, double bias,
    int limiter, int subcycles, int reinit, MHDMaterialParameters m1, MHDMaterialParameters m2) {
    double prm[5];
    mred_params(m1, m2, prm);
    std::vector<double> p = pack2(initialCells, 12, mint_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_MHD_INTERMEDIATE, p, (int)nx, (int)ny, prm, 5, dx, cfl, tEnd, bias, limiter, subcycles, 0, 2,
               reinit);
    return unpack2<MHDIntermediateStateVector>(p, nx, ny, 12, mint_make);
}

// --------------------------------------------------------------------------------------------- HPR solver
vector<HPRStateVector> HPRSecondOrderSolver::solve(vector<HPRStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                   double bias, int limiter, int subcycles, HPRMaterialParameters mp) {
    return solve(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, mp, 0);
}
vector<HPRStateVector> HPRSecondOrderSolver::solve(vector<HPRStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                   double bias, int limiter, int subcycles, HPRMaterialParameters mp,
                                                   int maxSteps) {
    double prm[20];
    hpr_params(mp, prm);
    std::vector<double> p = pack(initialCells, 17, hpr_get);
    run_planes(VG_MODEL_HPR, p, (int)initialCells.size(), 1, prm, 20, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps);
    return unpack<HPRStateVector>(p, initialCells.size(), 17, hpr_make);
}
vector<vector<HPRStateVector> > HPRSecondOrderSolver::solve2D(vector<vector<HPRStateVector> >& initialCells, double dx, double cfl,
                                                              double tEnd, double bias, int limiter, int subcycles,
                                                              HPRMaterialParameters mp) {
    return solve2D(initialCells, dx, cfl, tEnd, bias, limiter, subcycles, mp, 0);
}
vector<vector<HPRStateVector> > HPRSecondOrderSolver::solve2D(vector<vector<HPRStateVector> >& initialCells, double dx, double cfl,
                                                              double tEnd, double bias, int limiter, int subcycles,
                                                              HPRMaterialParameters mp, int maxSteps) {
    double prm[20];
    hpr_params(mp, prm);
    std::vector<double> p = pack2(initialCells, 17, hpr_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_HPR, p, (int)nx, (int)ny, prm, 20, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps);
    return unpack2<HPRStateVector>(p, nx, ny, 17, hpr_make);
}

// ------------------------------------------------------------------------------------------- first order
vector<EulerStateVector> FirstOrderSolver::solve(vector<EulerStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                 int subcycles, EulerMaterialParameters mp) {
    return solve(initialCells, dx, cfl, tEnd, subcycles, mp, 0);
}
vector<EulerStateVector> FirstOrderSolver::solve(vector<EulerStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                 int, EulerMaterialParameters mp, int maxSteps) {
    double prm[6];
    euler_params(mp, prm);
    std::vector<double> p = pack(initialCells, 6, euler_get);
    run_planes(VG_MODEL_EULER, p, (int)initialCells.size(), 1, prm, 6, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1);
    return unpack<EulerStateVector>(p, initialCells.size(), 6, euler_make);
}
vector<vector<EulerStateVector> > FirstOrderSolver::solve2D(vector<vector<EulerStateVector> >& initialCells, double dx,
                                                            double cfl, double tEnd, int subcycles, EulerMaterialParameters mp) {
    return solve2D(initialCells, dx, cfl, tEnd, subcycles, mp, 0);
}
vector<vector<EulerStateVector> > FirstOrderSolver::solve2D(vector<vector<EulerStateVector> >& initialCells, double dx,
                                                            double cfl, double tEnd, int, EulerMaterialParameters mp,
                                                            int maxSteps) {
    double prm[6];
    euler_params(mp, prm);
    std::vector<double> p = pack2(initialCells, 6, euler_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_EULER, p, (int)nx, (int)ny, prm, 6, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1);
    return unpack2<EulerStateVector>(p, nx, ny, 6, euler_make);
}

vector<MHDStateVector> MHDFirstOrderSolver::solve(vector<MHDStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                  int subcycles, MHDMaterialParameters mp) {
    return solve(initialCells, dx, cfl, tEnd, subcycles, mp, 0);
}
vector<MHDStateVector> MHDFirstOrderSolver::solve(vector<MHDStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                  int, MHDMaterialParameters mp, int maxSteps) {
    double prm[3];
    mhd_params(mp, prm);
    std::vector<double> p = pack(initialCells, 9, mhd_get);
    run_planes(VG_MODEL_MHD, p, (int)initialCells.size(), 1, prm, 3, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1);
    return unpack<MHDStateVector>(p, initialCells.size(), 9, mhd_make);
}
vector<vector<MHDStateVector> > MHDFirstOrderSolver::solve2D(vector<vector<MHDStateVector> >& initialCells, double dx,
                                                             double cfl, double tEnd, int subcycles, MHDMaterialParameters mp) {
    return solve2D(initialCells, dx, cfl, tEnd, subcycles, mp, 0);
}
vector<vector<MHDStateVector> > MHDFirstOrderSolver::solve2D(vector<vector<MHDStateVector> >& initialCells, double dx,
                                                             double cfl, double tEnd, int, MHDMaterialParameters mp,
                                                             int maxSteps) {
    double prm[3];
    mhd_params(mp, prm);
    std::vector<double> p = pack2(initialCells, 9, mhd_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_MHD, p, (int)nx, (int)ny, prm, 3, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1);
    return unpack2<MHDStateVector>(p, nx, ny, 9, mhd_make);
}

vector<HPRStateVector> HPRFirstOrderSolver::solve(vector<HPRStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                  int subcycles, HPRMaterialParameters mp) {
    return solve(initialCells, dx, cfl, tEnd, subcycles, mp, 0);
}
vector<HPRStateVector> HPRFirstOrderSolver::solve(vector<HPRStateVector>& initialCells, double dx, double cfl, double tEnd,
                                                  int, HPRMaterialParameters mp, int maxSteps) {
    double prm[20];
    hpr_params(mp, prm);
    std::vector<double> p = pack(initialCells, 17, hpr_get);
    run_planes(VG_MODEL_HPR, p, (int)initialCells.size(), 1, prm, 20, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1);
    return unpack<HPRStateVector>(p, initialCells.size(), 17, hpr_make);
}
vector<vector<HPRStateVector> > HPRFirstOrderSolver::solve2D(vector<vector<HPRStateVector> >& initialCells, double dx,
                                                             double cfl, double tEnd, int subcycles, HPRMaterialParameters mp) {
    return solve2D(initialCells, dx, cfl, tEnd, subcycles, mp, 0);
}
vector<vector<HPRStateVector> > HPRFirstOrderSolver::solve2D(vector<vector<HPRStateVector> >& initialCells, double dx,
                                                             double cfl, double tEnd, int, HPRMaterialParameters mp,
                                                             int maxSteps) {
    double prm[20];
    hpr_params(mp, prm);
    std::vector<double> p = pack2(initialCells, 17, hpr_get);
    long ny = initialCells.size(), nx = initialCells[0].size();
    run_planes(VG_MODEL_HPR, p, (int)nx, (int)ny, prm, 20, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1);
    return unpack2<HPRStateVector>(p, nx, ny, 17, hpr_make);
}

// ------------------------------------------------------------------------------- HPR two-material models
namespace {
vector<vector<double> > tensor_of(const double* a9) {
    vector<vector<double> > A(3, vector<double>(3));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = a9[3 * i + j];
    return A;
}
void tensor_into(const vector<vector<double> >& A, double* a9) {
    if (A.size() != 3 || A[0].size() != 3 || A[1].size() != 3 || A[2].size() != 3)
        throw std::invalid_argument("HPR: the distortion tensor must be 3x3");
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a9[3 * i + j] = A[i][j];
}
bool either_thermal(const HPRMaterialParameters& m1, const HPRMaterialParameters& m2) {
    return m1.getIsThermal() || m2.getIsThermal();
}
// each material's 20-value HPR block (hpr_params), material k at prm[20 k]: any equation of state, elastic or plastic
void hpr_two_params(const HPRMaterialParameters& m1, const HPRMaterialParameters& m2, double* prm) {
    hpr_params(m1, prm);
    hpr_params(m2, prm + 20);
}
void hred_get(const HPRReducedStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 19); }
HPRReducedStateVector hred_make(const double* w) {
    HPRReducedStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 19);
    return s;
}
void hint_get(const HPRIntermediateStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 20); }
HPRIntermediateStateVector hint_make(const double* w) {
    HPRIntermediateStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 20);
    return s;
}
// With neither material thermal, setConservedVariableVector leaves a cell's J alone, so every cell keeps the J it
// was given (the device, which never reads it then, carries zeros)
int heat_flux_plane(const HPRReducedStateVector&) { return 14; }
int heat_flux_plane(const HPRIntermediateStateVector&) { return 13; }
template <class S>
void keep_cold_heat_flux(S* out, const S* in, long n, const HPRMaterialParameters& m1, const HPRMaterialParameters& m2) {
    if (either_thermal(m1, m2)) return;
    for (long i = 0; i < n; i++) {
        const int j0 = heat_flux_plane(in[i]);
        for (int k = 0; k < 3; k++) out[i].data()[j0 + k] = in[i].data()[j0 + k];
    }
}
template <class S, class Get, class Make>
vector<S> hpr_two_run(int model, int nvar, vector<S>& cells, const HPRMaterialParameters& m1,
                      const HPRMaterialParameters& m2, double dx, double cfl, double tEnd, double bias, int limiter,
                      int subcycles, int maxSteps, int order, int reinit, Get get, Make make) {
    double prm[40];
    hpr_two_params(m1, m2, prm);
    std::vector<double> p = pack(cells, nvar, get);
    run_planes(model, p, (int)cells.size(), 1, prm, 40, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps, order,
               reinit);
    vector<S> out = unpack<S>(p, cells.size(), nvar, make);
    keep_cold_heat_flux(out.data(), cells.data(), (long)cells.size(), m1, m2);
    return out;
}
template <class S, class Get, class Make>
vector<vector<S> > hpr_two_run2(int model, int nvar, vector<vector<S> >& cells, const HPRMaterialParameters& m1,
                                const HPRMaterialParameters& m2, double dx, double cfl, double tEnd, double bias,
                                int limiter, int subcycles, int maxSteps, int order, int reinit, Get get, Make make) {
    double prm[40];
    hpr_two_params(m1, m2, prm);
    std::vector<double> p = pack2(cells, nvar, get);
    long ny = cells.size(), nx = cells[0].size();
    run_planes(model, p, (int)nx, (int)ny, prm, 40, dx, cfl, tEnd, bias, limiter, subcycles, maxSteps, order, reinit);
    vector<vector<S> > out = unpack2<S>(p, nx, ny, nvar, make);
    for (long i = 0; i < ny; i++) keep_cold_heat_flux(out[i].data(), cells[i].data(), nx, m1, m2);
    return out;
}
}  // namespace

// HPRReducedStateVector() (HPR/Multiphysics/hprreducedstatevector.cpp:3-19)
HPRReducedStateVector::HPRReducedStateVector()
    : w_{0.999, 1.0 / 1.4, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0} {}
HPRReducedStateVector::HPRReducedStateVector(double a1, double p, vector<vector<double> > A, double u, double v, double w,
                                             double jx, double jy, double jz, double r1, double r2)
    : w_{a1, p, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, u, v, w, jx, jy, jz, r1, r2} {
    tensor_into(A, w_ + 2);
}
void HPRReducedStateVector::setPrimitiveVariableVector(vector<double> w, HPRMaterialParameters m1,
                                                       HPRMaterialParameters m2) {
    const bool thermal = either_thermal(m1, m2);
    for (int i = 0; i < 19; i++)
        if (thermal || i < 14 || i > 16) w_[i] = w[i];
}
vector<double> HPRReducedStateVector::computePrimitiveVariableVector(HPRMaterialParameters m1,
                                                                     HPRMaterialParameters m2) const {
    vector<double> w(w_, w_ + 19);
    if (!either_thermal(m1, m2)) w[14] = w[15] = w[16] = 0.0;
    return w;
}
vector<vector<double> > HPRReducedStateVector::getInterfaceDistortionTensor() const { return tensor_of(w_ + 2); }

// HPRIntermediateStateVector() (HPR/Multiphysics/hprintermediatestatevector.cpp:3-21)
HPRIntermediateStateVector::HPRIntermediateStateVector()
    : w_{0.999, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0 / 1.4, 1.0, 1.0 / 1.4} {}
HPRIntermediateStateVector::HPRIntermediateStateVector(double a1, vector<vector<double> > A, double u, double v,
                                                       double w, double jx, double jy, double jz, double r1, double p1,
                                                       double r2, double p2)
    : w_{a1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, u, v, w, jx, jy, jz, r1, p1, r2, p2} {
    tensor_into(A, w_ + 1);
}
void HPRIntermediateStateVector::setPrimitiveVariableVector(vector<double> w, HPRMaterialParameters m1,
                                                            HPRMaterialParameters m2) {
    const bool thermal = either_thermal(m1, m2);
    for (int i = 0; i < 20; i++)
        if (thermal || i < 13 || i > 15) w_[i] = w[i];
}
vector<double> HPRIntermediateStateVector::computePrimitiveVariableVector(HPRMaterialParameters m1,
                                                                          HPRMaterialParameters m2) const {
    vector<double> w(w_, w_ + 20);
    if (!either_thermal(m1, m2)) w[13] = w[14] = w[15] = 0.0;
    return w;
}
vector<vector<double> > HPRIntermediateStateVector::getInterfaceDistortionTensor() const { return tensor_of(w_ + 1); }

vector<HPRReducedStateVector> HPRSecondOrderSolver::solve(vector<HPRReducedStateVector>& initialCells, double dx,
                                                          double cfl, double tEnd, double bias, int limiter,
                                                          int subcycles, int reinit, HPRMaterialParameters m1,
                                                          HPRMaterialParameters m2, int maxSteps) {
    return hpr_two_run(VG_MODEL_HPR_REDUCED, 19, initialCells, m1, m2, dx, cfl, tEnd, bias, limiter, subcycles,
                       maxSteps, 2, reinit, hred_get, hred_make);
}
vector<vector<HPRReducedStateVector> > HPRSecondOrderSolver::solve2D(vector<vector<HPRReducedStateVector> >& initialCells,
                                                                     double dx, double cfl, double tEnd, double bias,
                                                                     int limiter, int subcycles, int reinit,
                                                                     HPRMaterialParameters m1, HPRMaterialParameters m2,
                                                                     int maxSteps) {
    return hpr_two_run2(VG_MODEL_HPR_REDUCED, 19, initialCells, m1, m2, dx, cfl, tEnd, bias, limiter, subcycles,
                        maxSteps, 2, reinit, hred_get, hred_make);
}
vector<HPRIntermediateStateVector> HPRSecondOrderSolver::solve(vector<HPRIntermediateStateVector>& initialCells,
                                                               double dx, double cfl, double tEnd, double bias,
                                                               int limiter, int subcycles, int reinit,
                                                               HPRMaterialParameters m1, HPRMaterialParameters m2,
                                                               int maxSteps) {
    return hpr_two_run(VG_MODEL_HPR_INTERMEDIATE, 20, initialCells, m1, m2, dx, cfl, tEnd, bias, limiter, subcycles,
                       maxSteps, 2, reinit, hint_get, hint_make);
}
vector<vector<HPRIntermediateStateVector> > HPRSecondOrderSolver::solve2D(
    vector<vector<HPRIntermediateStateVector> >& initialCells, double dx, double cfl, double tEnd, double bias,
    int limiter, int subcycles, int reinit, HPRMaterialParameters m1, HPRMaterialParameters m2, int maxSteps) {
    return hpr_two_run2(VG_MODEL_HPR_INTERMEDIATE, 20, initialCells, m1, m2, dx, cfl, tEnd, bias, limiter, subcycles,
                        maxSteps, 2, reinit, hint_get, hint_make);
}
vector<HPRReducedStateVector> HPRFirstOrderSolver::solve(vector<HPRReducedStateVector>& initialCells, double dx,
                                                         double cfl, double tEnd, int, HPRMaterialParameters m1,
                                                         HPRMaterialParameters m2, int maxSteps) {
    return hpr_two_run(VG_MODEL_HPR_REDUCED, 19, initialCells, m1, m2, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1, 0,
                       hred_get, hred_make);
}
vector<vector<HPRReducedStateVector> > HPRFirstOrderSolver::solve2D(vector<vector<HPRReducedStateVector> >& initialCells,
                                                                    double dx, double cfl, double tEnd, int,
                                                                    HPRMaterialParameters m1, HPRMaterialParameters m2,
                                                                    int maxSteps) {
    return hpr_two_run2(VG_MODEL_HPR_REDUCED, 19, initialCells, m1, m2, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1, 0,
                        hred_get, hred_make);
}
vector<HPRIntermediateStateVector> HPRFirstOrderSolver::solve(vector<HPRIntermediateStateVector>& initialCells,
                                                              double dx, double cfl, double tEnd, int,
                                                              HPRMaterialParameters m1, HPRMaterialParameters m2,
                                                              int maxSteps) {
    return hpr_two_run(VG_MODEL_HPR_INTERMEDIATE, 20, initialCells, m1, m2, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1, 0,
                       hint_get, hint_make);
}
vector<vector<HPRIntermediateStateVector> > HPRFirstOrderSolver::solve2D(
    vector<vector<HPRIntermediateStateVector> >& initialCells, double dx, double cfl, double tEnd, int,
    HPRMaterialParameters m1, HPRMaterialParameters m2, int maxSteps) {
    return hpr_two_run2(VG_MODEL_HPR_INTERMEDIATE, 20, initialCells, m1, m2, dx, cfl, tEnd, 0.0, 0, 0, maxSteps, 1, 0,
                        hint_get, hint_make);
}

// ---------------------------------------------------------------------------------- HPR multiphysics model
namespace {
void hmph_get(const HPRMultiphysicsStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 32); }
HPRMultiphysicsStateVector hmph_make(const double* w) {
    HPRMultiphysicsStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 32);
    return s;
}
}  // namespace

// HPRMultiphysicsStateVector() (HPR/Multiphysics/hprmultiphysicsstatevector.cpp:3-26)
HPRMultiphysicsStateVector::HPRMultiphysicsStateVector() : w_{} {
    w_[0] = 0.999;
    for (int k = 0; k < 2; k++) {
        w_[4 + 14 * k] = 1.0;
        w_[5 + 14 * k] = 1.0 / 1.4;
        w_[6 + 14 * k] = w_[10 + 14 * k] = w_[14 + 14 * k] = 1.0;
    }
}
HPRMultiphysicsStateVector::HPRMultiphysicsStateVector(double a1, double u, double v, double w, double r1, double p1,
                                                       vector<vector<double> > A1, double j1x, double j1y, double j1z,
                                                       double r2, double p2, vector<vector<double> > A2, double j2x,
                                                       double j2y, double j2z)
    : w_{} {
    const double head[6] = {a1, u, v, w, r1, p1};
    for (int i = 0; i < 6; i++) w_[i] = head[i];
    tensor_into(A1, w_ + 6);
    w_[15] = j1x, w_[16] = j1y, w_[17] = j1z;
    w_[18] = r2, w_[19] = p2;
    tensor_into(A2, w_ + 20);
    w_[29] = j2x, w_[30] = j2y, w_[31] = j2z;
}
void HPRMultiphysicsStateVector::setPrimitiveVariableVector(vector<double> w, HPRMaterialParameters m1,
                                                            HPRMaterialParameters m2) {
    for (int i = 0; i < 32; i++) {
        if (i >= 15 && i < 18 && !m1.getIsThermal()) continue;
        if (i >= 29 && !m2.getIsThermal()) continue;
        w_[i] = w[i];
    }
}
vector<double> HPRMultiphysicsStateVector::computePrimitiveVariableVector(HPRMaterialParameters m1,
                                                                          HPRMaterialParameters m2) const {
    vector<double> w(w_, w_ + 32);
    if (!m1.getIsThermal()) w[15] = w[16] = w[17] = 0.0;
    if (!m2.getIsThermal()) w[29] = w[30] = w[31] = 0.0;
    return w;
}
vector<vector<double> > HPRMultiphysicsStateVector::getMaterial1DistortionTensor() const { return tensor_of(w_ + 6); }
vector<vector<double> > HPRMultiphysicsStateVector::getMaterial2DistortionTensor() const { return tensor_of(w_ + 20); }

vector<HPRMultiphysicsStateVector> HPRSecondOrderSolver::solve(vector<HPRMultiphysicsStateVector>& initialCells,
                                                               double dx, double cfl, double tEnd, double bias,
                                                               int limiter, int subcycles, int reinit,
                                                               HPRMaterialParameters m1, HPRMaterialParameters m2,
                                                               int maxSteps) {
    double prm[40];
    hpr_two_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 32, hmph_get);
    run_planes(VG_MODEL_HPR_MULTIPHYSICS, p, (int)initialCells.size(), 1, prm, 40, dx, cfl, tEnd, bias, limiter,
               subcycles, maxSteps, 2, reinit);
    return unpack<HPRMultiphysicsStateVector>(p, initialCells.size(), 32, hmph_make);
}
vector<HPRMultiphysicsStateVector> HPRFirstOrderSolver::solve(vector<HPRMultiphysicsStateVector>& initialCells,
                                                              double dx, double cfl, double tEnd, int,
                                                              HPRMaterialParameters m1, HPRMaterialParameters m2,
                                                              int maxSteps) {
    double prm[40];
    hpr_two_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 32, hmph_get);
    run_planes(VG_MODEL_HPR_MULTIPHYSICS, p, (int)initialCells.size(), 1, prm, 40, dx, cfl, tEnd, 0.0, 0, 0, maxSteps,
               1, 0);
    return unpack<HPRMultiphysicsStateVector>(p, initialCells.size(), 32, hmph_make);
}

// ---------------------------------------------------------------------------------- MHD multiphysics model
// MHDMultiphysicsStateVector() (MHD/Multiphysics/mhdmultiphysicsstatevector.cpp:3-27)
MHDMultiphysicsStateVector::MHDMultiphysicsStateVector()
    : w_{0.999, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0} {}
MHDMultiphysicsStateVector::MHDMultiphysicsStateVector(double a1, double u, double v, double w, double r1, double p1,
                                                       double b1x, double b1y, double b1z, double psi1, double r2,
                                                       double p2, double b2x, double b2y, double b2z, double psi2)
    : w_{a1, u, v, w, r1, p1, b1x, b1y, b1z, psi1, r2, p2, b2x, b2y, b2z, psi2} {}
void MHDMultiphysicsStateVector::setPrimitiveVariableVector(vector<double> w) {
    for (int i = 0; i < 16; i++) w_[i] = w[i];
}

namespace {
void mmph_get(const MHDMultiphysicsStateVector& c, double* w) { std::memcpy(w, c.data(), sizeof(double) * 16); }
MHDMultiphysicsStateVector mmph_make(const double* w) {
    MHDMultiphysicsStateVector s;
    std::memcpy(s.data(), w, sizeof(double) * 16);
    return s;
}
// {gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2}
void mmph_params(const MHDMaterialParameters& m1, const MHDMaterialParameters& m2, double* prm) {
    prm[0] = m1.getAdiabaticIndex(), prm[1] = m1.getStiffeningParameter();
    prm[2] = m2.getAdiabaticIndex(), prm[3] = m2.getStiffeningParameter();
    prm[4] = m1.getHyperbolicWaveSpeed(), prm[5] = m2.getHyperbolicWaveSpeed();
}
}  // namespace

vector<MHDMultiphysicsStateVector> MHDSecondOrderSolver::solve(vector<MHDMultiphysicsStateVector>& initialCells,
                                                               double dx, double cfl, double tEnd, double bias,
                                                               int limiter, int subcycles, int reinit,
                                                               MHDMaterialParameters m1, MHDMaterialParameters m2,
                                                               int maxSteps) {
    double prm[6];
    mmph_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 16, mmph_get);
    run_planes(VG_MODEL_MHD_MULTIPHYSICS, p, (int)initialCells.size(), 1, prm, 6, dx, cfl, tEnd, bias, limiter,
               subcycles, maxSteps, 2, reinit);
    return unpack<MHDMultiphysicsStateVector>(p, initialCells.size(), 16, mmph_make);
}
vector<MHDMultiphysicsStateVector> MHDFirstOrderSolver::solve(vector<MHDMultiphysicsStateVector>& initialCells,
                                                              double dx, double cfl, double tEnd, int,
                                                              MHDMaterialParameters m1, MHDMaterialParameters m2,
                                                              int maxSteps) {
    double prm[6];
    mmph_params(m1, m2, prm);
    std::vector<double> p = pack(initialCells, 16, mmph_get);
    run_planes(VG_MODEL_MHD_MULTIPHYSICS, p, (int)initialCells.size(), 1, prm, 6, dx, cfl, tEnd, 0.0, 0, 0, maxSteps,
               1, 0);
    return unpack<MHDMultiphysicsStateVector>(p, initialCells.size(), 16, mmph_make);
}
