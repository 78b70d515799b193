// Drop-in C++ surface of Vanguard's single-material SLIC path, backed by the B200 C ABI (include/vanguard_slic.h).
//
// Same class names, static-method signatures and value semantics as the reference's Solvers/ entry points
// (Solvers/secondordersolver.h:7-72, Solvers/mhdsecondordersolver.h:12-70, Solvers/hprsecondordersolver.h:12-67,
// Solvers/slopelimiters.h:23-70, Solvers/solvers.h:8-76) and of the model types they take, so existing callers
// recompile against vanguard_b200/shim and link libvanguard_shim.so instead of the OpenMP sources:
//   * solve / solve2D copy the input, run the whole time loop on the GPU and return the result by value;
//   * the per-sweep functions update `cells` in place from the caller's ghosted array;
//   * errors (no GPU, unsupported input) throw std::runtime_error with the C ABI's message -- the reference has
//     no error reporting, and this layer never falls back to a CPU path.
// Environment: VG_DEVICE selects the CUDA device (default 0); VG_PRECISION=mixed selects the mixed FP32/FP64 form
// (default: the plain FP64 form, bitwise equal to the reference).
#pragma once

#include <string>
#include <vector>

using std::string;
using std::vector;

// ------------------------------------------------------------------------------------------------- Euler
class EulerMaterialParameters {
public:
    EulerMaterialParameters();
    explicit EulerMaterialParameters(double newAdiabaticIndex);
    EulerMaterialParameters(double newAdiabaticIndex, double newStiffeningParameter);
    EulerMaterialParameters(double newAdiabaticIndex, double newStiffeningParameter, double newSpecificHeatCapacity,
                            double newEnergyOfFormation, double newIgnitionTemperature, double newReactionRate);
    void setAdiabaticIndex(double v) { adiabaticIndex = v; }
    void setStiffeningParameter(double v) { stiffeningParameter = v; }
    void setSpecificHeatCapacity(double v) { specificHeatCapacity = v; }
    void setEnergyOfFormation(double v) { energyOfFormation = v; }
    void setIgnitionTemperature(double v) { ignitionTemperature = v; }
    void setReactionRate(double v) { reactionRate = v; }
    double getAdiabaticIndex() const { return adiabaticIndex; }
    double getStiffeningParameter() const { return stiffeningParameter; }
    double getSpecificHeatCapacity() const { return specificHeatCapacity; }
    double getEnergyOfFormation() const { return energyOfFormation; }
    double getIgnitionTemperature() const { return ignitionTemperature; }
    double getReactionRate() const { return reactionRate; }

private:
    double adiabaticIndex, stiffeningParameter, specificHeatCapacity, energyOfFormation, ignitionTemperature, reactionRate;
};

class EulerEquationOfState {
public:
    static double computeSpecificInternalEnergy(double density, double pressure, EulerMaterialParameters mp);
    static double computePressure(double density, double specificInternalEnergy, EulerMaterialParameters mp);
    static double computeSoundSpeed(double density, double pressure, EulerMaterialParameters mp);
};

class EulerStateVector {
public:
    EulerStateVector();
    EulerStateVector(double newDensity, double newXVelocity, double newYVelocity, double newZVelocity, double newPressure);
    EulerStateVector(double newDensity, double newXVelocity, double newYVelocity, double newZVelocity, double newPressure,
                     double newReactionProgress);
    void setPrimitiveVariableVector(vector<double> w);
    void setConservedVariableVector(vector<double> u, EulerMaterialParameters mp);
    vector<double> computePrimitiveVariableVector() const;
    vector<double> computeConservedVariableVector(EulerMaterialParameters mp) const;
    static vector<double> computeXFluxVector(vector<double> u, EulerMaterialParameters mp);
    vector<double> computeXFluxVector(EulerMaterialParameters mp) const;
    static vector<double> computeYFluxVector(vector<double> u, EulerMaterialParameters mp);
    vector<double> computeYFluxVector(EulerMaterialParameters mp) const;
    double computeSpecificInternalEnergy(EulerMaterialParameters mp) const;
    double computeTotalEnergy(EulerMaterialParameters mp) const;
    double computeSoundSpeed(EulerMaterialParameters mp) const;
    void setDensity(double v) { density = v; }
    void setXVelocity(double v) { xVelocity = v; }
    void setYVelocity(double v) { yVelocity = v; }
    void setZVelocity(double v) { zVelocity = v; }
    void setPressure(double v) { pressure = v; }
    void setReactionProgress(double v) { reactionProgress = v; }
    double getDensity() const { return density; }
    double getXVelocity() const { return xVelocity; }
    double getYVelocity() const { return yVelocity; }
    double getZVelocity() const { return zVelocity; }
    double getPressure() const { return pressure; }
    double getReactionProgress() const { return reactionProgress; }

private:
    double density, xVelocity, yVelocity, zVelocity, pressure, reactionProgress;
};

// EulerReducedStateVector (Euler/Multiphysics/eulerreducedstatevector.h): the reduced two-material state,
// primitives alpha1, u, v, w, rho1, rho2, p.
class EulerReducedStateVector {
public:
    EulerReducedStateVector();
    EulerReducedStateVector(double newMaterial1VolumeFraction, double newInterfaceXVelocity, double newInterfaceYVelocity,
                            double newInterfaceZVelocity, double newMaterial1Density, double newMaterial2Density,
                            double newInterfacePressure);
    void setPrimitiveVariableVector(vector<double> w);
    vector<double> computePrimitiveVariableVector() const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getInterfaceXVelocity() const { return w_[1]; }
    double getInterfaceYVelocity() const { return w_[2]; }
    double getInterfaceZVelocity() const { return w_[3]; }
    double getMaterial1Density() const { return w_[4]; }
    double getMaterial2Density() const { return w_[5]; }
    double getInterfacePressure() const { return w_[6]; }
    void setMaterial1VolumeFraction(double v) { w_[0] = v; }
    void setInterfaceXVelocity(double v) { w_[1] = v; }
    void setInterfaceYVelocity(double v) { w_[2] = v; }
    void setInterfaceZVelocity(double v) { w_[3] = v; }
    void setMaterial1Density(double v) { w_[4] = v; }
    void setMaterial2Density(double v) { w_[5] = v; }
    void setInterfacePressure(double v) { w_[6] = v; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[7];
};

// EulerMultiphysicsStateVector (Euler/Multiphysics/eulermultiphysicsstatevector.h): the multiphysics two-material
// state, primitives alpha1, u, v, w, rho1, p1, rho2, p2.
class EulerMultiphysicsStateVector {
public:
    EulerMultiphysicsStateVector();
    EulerMultiphysicsStateVector(double newMaterial1VolumeFraction, double newInterfaceXVelocity, double newInterfaceYVelocity,
                                 double newInterfaceZVelocity, double newMaterial1Density, double newMaterial1Pressure,
                                 double newMaterial2Density, double newMaterial2Pressure);
    void setPrimitiveVariableVector(vector<double> w);
    vector<double> computePrimitiveVariableVector() const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getInterfaceXVelocity() const { return w_[1]; }
    double getInterfaceYVelocity() const { return w_[2]; }
    double getInterfaceZVelocity() const { return w_[3]; }
    double getMaterial1Density() const { return w_[4]; }
    double getMaterial1Pressure() const { return w_[5]; }
    double getMaterial2Density() const { return w_[6]; }
    double getMaterial2Pressure() const { return w_[7]; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[8];
};

// --------------------------------------------------------------------------------------------------- MHD
class MHDMaterialParameters {
public:
    MHDMaterialParameters();
    explicit MHDMaterialParameters(double newAdiabaticIndex);
    double computeHyperbolicWaveSpeedSquared() const { return hyperbolicWaveSpeed * hyperbolicWaveSpeed; }
    double computeParabolicDampingSquared() const { return parabolicDamping * parabolicDamping; }
    void configureParabolicDamping();
    void setAdiabaticIndex(double v) { adiabaticIndex = v; }
    void setStiffeningParameter(double v) { stiffeningParameter = v; }
    void setHyperbolicWaveSpeed(double v) { hyperbolicWaveSpeed = v; }
    void setParabolicDamping(double v) { parabolicDamping = v; }
    double getAdiabaticIndex() const { return adiabaticIndex; }
    double getStiffeningParameter() const { return stiffeningParameter; }
    double getHyperbolicWaveSpeed() const { return hyperbolicWaveSpeed; }
    double getParabolicDamping() const { return parabolicDamping; }

private:
    double adiabaticIndex, stiffeningParameter, hyperbolicWaveSpeed, parabolicDamping;
};

class MHDStateVector {
public:
    MHDStateVector();
    MHDStateVector(double newDensity, double newXVelocity, double newYVelocity, double newZVelocity, double newPressure,
                   double newXMagneticField, double newYMagneticField, double newZMagneticField, double newAuxiliaryField);
    void setPrimitiveVariableVector(vector<double> w);
    vector<double> computePrimitiveVariableVector() const;
    vector<double> computeConservedVariableVector(MHDMaterialParameters mp) const;
    void setConservedVariableVector(vector<double> u, MHDMaterialParameters mp);
    double getDensity() const { return w_[0]; }
    double getXVelocity() const { return w_[1]; }
    double getYVelocity() const { return w_[2]; }
    double getZVelocity() const { return w_[3]; }
    double getPressure() const { return w_[4]; }
    double getXMagneticField() const { return w_[5]; }
    double getYMagneticField() const { return w_[6]; }
    double getZMagneticField() const { return w_[7]; }
    double getAuxiliaryField() const { return w_[8]; }
    void setDensity(double v) { w_[0] = v; }
    void setXVelocity(double v) { w_[1] = v; }
    void setYVelocity(double v) { w_[2] = v; }
    void setZVelocity(double v) { w_[3] = v; }
    void setPressure(double v) { w_[4] = v; }
    void setXMagneticField(double v) { w_[5] = v; }
    void setYMagneticField(double v) { w_[6] = v; }
    void setZMagneticField(double v) { w_[7] = v; }
    void setAuxiliaryField(double v) { w_[8] = v; }

private:
    double w_[9];
};

// MHDReducedStateVector (MHD/Multiphysics/mhdreducedstatevector.h): the MHD reduced two-material state, primitives
// alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi.
class MHDReducedStateVector {
public:
    MHDReducedStateVector();
    MHDReducedStateVector(double newMaterial1VolumeFraction, double newInterfaceXVelocity, double newInterfaceYVelocity,
                          double newInterfaceZVelocity, double newMaterial1Density, double newMaterial2Density,
                          double newInterfacePressure, double newInterfaceXMagneticField,
                          double newInterfaceYMagneticField, double newInterfaceZMagneticField,
                          double newInterfaceAuxiliaryField);
    void setPrimitiveVariableVector(vector<double> w);
    vector<double> computePrimitiveVariableVector() const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getInterfaceXVelocity() const { return w_[1]; }
    double getInterfaceYVelocity() const { return w_[2]; }
    double getInterfaceZVelocity() const { return w_[3]; }
    double getMaterial1Density() const { return w_[4]; }
    double getMaterial2Density() const { return w_[5]; }
    double getInterfacePressure() const { return w_[6]; }
    double getInterfaceXMagneticField() const { return w_[7]; }
    double getInterfaceYMagneticField() const { return w_[8]; }
    double getInterfaceZMagneticField() const { return w_[9]; }
    double getInterfaceAuxiliaryField() const { return w_[10]; }
    void setMaterial1VolumeFraction(double v) { w_[0] = v; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[11];
};

// MHDIntermediateStateVector (MHD/Multiphysics/mhdintermediatestatevector.h): the MHD intermediate two-material state,
// primitives alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi.
class MHDIntermediateStateVector {
public:
    MHDIntermediateStateVector();
    void setPrimitiveVariableVector(vector<double> w);
    vector<double> computePrimitiveVariableVector() const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getMaterial1Density() const { return w_[4]; }
    double getMaterial1Pressure() const { return w_[5]; }
    double getMaterial2Density() const { return w_[6]; }
    double getMaterial2Pressure() const { return w_[7]; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[12];
};

// MHDMultiphysicsStateVector (MHD/Multiphysics/mhdmultiphysicsstatevector.h; 1D): the MHD multiphysics two-material
// state, primitives alpha1, u, v, w, rho1, p1, B1 (3), psi1, rho2, p2, B2 (3), psi2.
class MHDMultiphysicsStateVector {
public:
    MHDMultiphysicsStateVector();
    MHDMultiphysicsStateVector(double newMaterial1VolumeFraction, double newInterfaceXVelocity,
                               double newInterfaceYVelocity, double newInterfaceZVelocity, double newMaterial1Density,
                               double newMaterial1Pressure, double newMaterial1XMagneticField,
                               double newMaterial1YMagneticField, double newMaterial1ZMagneticField,
                               double newMaterial1AuxiliaryField, double newMaterial2Density, double newMaterial2Pressure,
                               double newMaterial2XMagneticField, double newMaterial2YMagneticField,
                               double newMaterial2ZMagneticField, double newMaterial2AuxiliaryField);
    void setPrimitiveVariableVector(vector<double> w);
    vector<double> computePrimitiveVariableVector() const { return vector<double>(w_, w_ + 16); }
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getInterfaceXVelocity() const { return w_[1]; }
    double getMaterial1Density() const { return w_[4]; }
    double getMaterial1Pressure() const { return w_[5]; }
    double getMaterial2Density() const { return w_[10]; }
    double getMaterial2Pressure() const { return w_[11]; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[16];
};

// --------------------------------------------------------------------------------------------------- HPR
class HPRMaterialParameters {
public:
    HPRMaterialParameters();
    HPRMaterialParameters(string newEquationOfState, bool newIsThermal, bool newIsPlastic, double newIdealGasConstant,
                          double newReferenceDensity, double newReferencePressure, double newReferenceTemperature,
                          double newInitialTemperature, double newSpecificHeatCapacity, double newAdiabaticIndex,
                          double newStiffeningParameter, double newReferenceSoundSpeed, double newReferenceGruneisenCoefficient,
                          double newHugoniotSlopeCoefficient, double newReferenceInternalEnergy, double newTransverseWaveSpeed,
                          double newStrainDissipationTime, double newThermalImpulseRelaxationTime,
                          double newDynamicViscosityCoefficient, double newPrandtlNumber,
                          double newElasticPlasticTransitionParameter, double newPowerLawIndex, double newHeatWaveSpeed,
                          double newAlphaParameter, double newBetaParameter, double newGammaParameter);
    void configureStrainDissipationTime();
    void configureThermalImpulseRelaxationTime();
    void configureThermalImpulseRelaxationTime(double heatConductionCoefficient);
    double computeStrainDissipationTime() const;
    double computeHeatConductionCoefficient() const;
    double computeThermalImpulseRelaxationTime() const;
    double computeThermalImpulseRelaxationTime(double heatConductionCoefficient) const;
    string getEquationOfState() const { return equationOfState; }
    bool getIsThermal() const { return isThermal; }
    bool getIsPlastic() const { return isPlastic; }
    double getReferenceDensity() const { return referenceDensity; }
    double getReferencePressure() const { return referencePressure; }
    double getReferenceTemperature() const { return referenceTemperature; }
    double getInitialTemperature() const { return initialTemperature; }
    double getSpecificHeatCapacity() const { return specificHeatCapacity; }
    double getAdiabaticIndex() const { return adiabaticIndex; }
    double getStiffeningParameter() const { return stiffeningParameter; }
    double getTransverseWaveSpeed() const { return transverseWaveSpeed; }
    double getStrainDissipationTime() const { return strainDissipationTime; }
    double getThermalImpulseRelaxationTime() const { return thermalImpulseRelaxationTime; }
    double getHeatWaveSpeed() const { return heatWaveSpeed; }
    double getReferenceSoundSpeed() const { return referenceSoundSpeed; }
    double getReferenceGruneisenCoefficient() const { return referenceGruneisenCoefficient; }
    double getHugoniotSlopeCoefficient() const { return hugoniotSlopeCoefficient; }
    double getElasticPlasticTransitionParameter() const { return elasticPlasticTransitionParameter; }
    double getPowerLawIndex() const { return powerLawIndex; }
    double getAlphaParameter() const { return alphaParameter; }
    void setIsThermal(bool v) { isThermal = v; }
    void setStrainDissipationTime(double v) { strainDissipationTime = v; }
    void setThermalImpulseRelaxationTime(double v) { thermalImpulseRelaxationTime = v; }

private:
    string equationOfState;
    bool isThermal, isPlastic;
    double idealGasConstant, referenceDensity, referencePressure, referenceTemperature, initialTemperature,
        specificHeatCapacity, adiabaticIndex, stiffeningParameter, referenceSoundSpeed, referenceGruneisenCoefficient,
        hugoniotSlopeCoefficient, referenceInternalEnergy, transverseWaveSpeed, strainDissipationTime,
        thermalImpulseRelaxationTime, dynamicViscosityCoefficient, prandtlNumber, elasticPlasticTransitionParameter,
        powerLawIndex, heatWaveSpeed, alphaParameter, betaParameter, gammaParameter;
};

class HPRStateVector {
public:
    HPRStateVector();
    HPRStateVector(double newDensity, double newPressure, vector<vector<double> > newDistortionTensor, double newXVelocity,
                   double newYVelocity, double newZVelocity, double newXThermalImpulse, double newYThermalImpulse,
                   double newZThermalImpulse);
    double getDensity() const { return w_[0]; }
    double getPressure() const { return w_[1]; }
    vector<vector<double> > getDistortionTensor() const;
    double getXVelocity() const { return w_[11]; }
    double getYVelocity() const { return w_[12]; }
    double getZVelocity() const { return w_[13]; }
    double getXThermalImpulse() const { return w_[14]; }
    double getYThermalImpulse() const { return w_[15]; }
    double getZThermalImpulse() const { return w_[16]; }
    void setDensity(double v) { w_[0] = v; }
    void setPressure(double v) { w_[1] = v; }
    void setDistortionTensor(vector<vector<double> > a);
    void setXVelocity(double v) { w_[11] = v; }
    void setYVelocity(double v) { w_[12] = v; }
    void setZVelocity(double v) { w_[13] = v; }
    void setXThermalImpulse(double v) { w_[14] = v; }
    void setYThermalImpulse(double v) { w_[15] = v; }
    void setZThermalImpulse(double v) { w_[16] = v; }
    const double* data() const { return w_; }
    double* data() { return w_; }

private:
    double w_[17];
};

// ------------------------------------------------------------------------------------------- slope limiters
// HPRReducedStateVector (HPR/Multiphysics/hprreducedstatevector.h): the HPR reduced two-material state, primitives
// alpha1, p, A (9, row-major), u, v, w, Jx, Jy, Jz, rho1, rho2.  As in the reference, the heat flux J is taken and
// returned only when either material is thermal (hprreducedstatevector.cpp:78-109, :154-185).
class HPRReducedStateVector {
public:
    HPRReducedStateVector();
    HPRReducedStateVector(double newMaterial1VolumeFraction, double newInterfacePressure,
                          vector<vector<double> > newInterfaceDistortionTensor, double newInterfaceXVelocity,
                          double newInterfaceYVelocity, double newInterfaceZVelocity, double newInterfaceXThermalImpulse,
                          double newInterfaceYThermalImpulse, double newInterfaceZThermalImpulse,
                          double newMaterial1Density, double newMaterial2Density);
    void setPrimitiveVariableVector(vector<double> w, HPRMaterialParameters material1Parameters,
                                    HPRMaterialParameters material2Parameters);
    vector<double> computePrimitiveVariableVector(HPRMaterialParameters material1Parameters,
                                                  HPRMaterialParameters material2Parameters) const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getInterfacePressure() const { return w_[1]; }
    vector<vector<double> > getInterfaceDistortionTensor() const;
    double getInterfaceXVelocity() const { return w_[11]; }
    double getInterfaceYVelocity() const { return w_[12]; }
    double getInterfaceZVelocity() const { return w_[13]; }
    double getInterfaceXThermalImpulse() const { return w_[14]; }
    double getInterfaceYThermalImpulse() const { return w_[15]; }
    double getInterfaceZThermalImpulse() const { return w_[16]; }
    double getMaterial1Density() const { return w_[17]; }
    double getMaterial2Density() const { return w_[18]; }
    void setMaterial1VolumeFraction(double v) { w_[0] = v; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[19];
};

// HPRIntermediateStateVector (HPR/Multiphysics/hprintermediatestatevector.h): the HPR intermediate two-material state,
// primitives alpha1, A (9, row-major), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2; J as for the reduced state
// (hprintermediatestatevector.cpp:82-110, :161-193).
class HPRIntermediateStateVector {
public:
    HPRIntermediateStateVector();
    HPRIntermediateStateVector(double newMaterial1VolumeFraction, vector<vector<double> > newInterfaceDistortionTensor,
                               double newInterfaceXVelocity, double newInterfaceYVelocity, double newInterfaceZVelocity,
                               double newInterfaceXThermalImpulse, double newInterfaceYThermalImpulse,
                               double newInterfaceZThermalImpulse, double newMaterial1Density, double newMaterial1Pressure,
                               double newMaterial2Density, double newMaterial2Pressure);
    void setPrimitiveVariableVector(vector<double> w, HPRMaterialParameters material1Parameters,
                                    HPRMaterialParameters material2Parameters);
    vector<double> computePrimitiveVariableVector(HPRMaterialParameters material1Parameters,
                                                  HPRMaterialParameters material2Parameters) const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    vector<vector<double> > getInterfaceDistortionTensor() const;
    double getInterfaceXVelocity() const { return w_[10]; }
    double getInterfaceYVelocity() const { return w_[11]; }
    double getInterfaceZVelocity() const { return w_[12]; }
    double getInterfaceXThermalImpulse() const { return w_[13]; }
    double getInterfaceYThermalImpulse() const { return w_[14]; }
    double getInterfaceZThermalImpulse() const { return w_[15]; }
    double getMaterial1Density() const { return w_[16]; }
    double getMaterial1Pressure() const { return w_[17]; }
    double getMaterial2Density() const { return w_[18]; }
    double getMaterial2Pressure() const { return w_[19]; }
    void setMaterial1VolumeFraction(double v) { w_[0] = v; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[20];
};

// HPRMultiphysicsStateVector (HPR/Multiphysics/hprmultiphysicsstatevector.h; 1D): the HPR multiphysics two-material
// state, primitives alpha1, u, v, w, rho1, p1, A1 (9), J1 (3), rho2, p2, A2 (9), J2 (3).  A material's J is taken and
// returned only when that material is thermal (hprmultiphysicsstatevector.cpp:98-139, :204-249); a cold material's J
// enters the solve as 0.
class HPRMultiphysicsStateVector {
public:
    HPRMultiphysicsStateVector();
    HPRMultiphysicsStateVector(double newMaterial1VolumeFraction, double newInterfaceXVelocity,
                               double newInterfaceYVelocity, double newInterfaceZVelocity, double newMaterial1Density,
                               double newMaterial1Pressure, vector<vector<double> > newMaterial1DistortionTensor,
                               double newMaterial1XThermalImpulse, double newMaterial1YThermalImpulse,
                               double newMaterial1ZThermalImpulse, double newMaterial2Density, double newMaterial2Pressure,
                               vector<vector<double> > newMaterial2DistortionTensor, double newMaterial2XThermalImpulse,
                               double newMaterial2YThermalImpulse, double newMaterial2ZThermalImpulse);
    void setPrimitiveVariableVector(vector<double> w, HPRMaterialParameters material1Parameters,
                                    HPRMaterialParameters material2Parameters);
    vector<double> computePrimitiveVariableVector(HPRMaterialParameters material1Parameters,
                                                  HPRMaterialParameters material2Parameters) const;
    double getMaterial1VolumeFraction() const { return w_[0]; }
    double getInterfaceXVelocity() const { return w_[1]; }
    double getInterfaceYVelocity() const { return w_[2]; }
    double getInterfaceZVelocity() const { return w_[3]; }
    double getMaterial1Density() const { return w_[4]; }
    double getMaterial1Pressure() const { return w_[5]; }
    vector<vector<double> > getMaterial1DistortionTensor() const;
    double getMaterial2Density() const { return w_[18]; }
    double getMaterial2Pressure() const { return w_[19]; }
    vector<vector<double> > getMaterial2DistortionTensor() const;
    void setMaterial1VolumeFraction(double v) { w_[0] = v; }
    double* data() { return w_; }
    const double* data() const { return w_; }

private:
    double w_[32];
};

class SlopeLimiters {
public:
    static double computeRCoefficient(double steepness, double bias);
    static double computeSuperBeeSlopeLimiter(double steepness, double bias);
    static double computeVanLeerSlopeLimiter(double steepness, double bias);
    static double computeMinBeeSlopeLimiter(double steepness, double bias);
    static double computeSlopeLimiter(double steepness, double bias, int slopeLimiter);
};

// ------------------------------------------------------------------------------------------- solver helpers
class Solvers {
public:
    static vector<EulerStateVector> insertBoundaryCells(vector<EulerStateVector>& currentCells, int boundarySize);
    static vector<vector<EulerStateVector> > insertBoundaryCells2D(vector<vector<EulerStateVector> >& currentCells, int boundarySize);
    static double computeMaximumWaveSpeed(vector<EulerStateVector>& currentCells, EulerMaterialParameters mp);
    static double computeMaximumWaveSpeed2D(vector<vector<EulerStateVector> >& currentCells, EulerMaterialParameters mp);
    static double computeStableTimeStep(vector<EulerStateVector>& currentCells, double cellSpacing, double CFLCoefficient,
                                        double currentTime, double finalTime, int currentIteration, EulerMaterialParameters mp);
    static double computeStableTimeStep2D(vector<vector<EulerStateVector> >& currentCells, double cellSpacing,
                                          double CFLCoefficient, double currentTime, double finalTime, int currentIteration,
                                          EulerMaterialParameters mp);
    static double computeStableTimeStep(double timeStep, double currentTime, double finalTime, int currentIteration);
};

// ------------------------------------------------------------------------------------------------ solvers
class SecondOrderSolver {
public:
    static void computeSLICTimeStep(vector<EulerStateVector>& currentCells, vector<EulerStateVector>& currentCellsWithBoundary,
                                    double cellSpacing, double timeStep, double bias, int slopeLimiter, EulerMaterialParameters mp);
    static void computeXSLICTimeStep2D(vector<vector<EulerStateVector> >& currentCells,
                                       vector<vector<EulerStateVector> >& currentCellsWithBoundary, double cellSpacing,
                                       double timeStep, double bias, int slopeLimiter, EulerMaterialParameters mp);
    static void computeYSLICTimeStep2D(vector<vector<EulerStateVector> >& currentCells,
                                       vector<vector<EulerStateVector> >& currentCellsWithBoundary, double cellSpacing,
                                       double timeStep, double bias, int slopeLimiter, EulerMaterialParameters mp);
    static vector<EulerStateVector> solve(vector<EulerStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                          double finalTime, double bias, int slopeLimiter, int subcyclingIterations,
                                          EulerMaterialParameters mp);
    static vector<vector<EulerStateVector> > solve2D(vector<vector<EulerStateVector> >& initialCells, double cellSpacing,
                                                     double CFLCofficient, double finalTime, double bias, int slopeLimiter,
                                                     int subcyclingIterations, EulerMaterialParameters mp);
    // the reduced two-material model (Solvers/secondordersolver.cpp:354-385, :470-...): reinitialisationFrequency > 0
    // reinitialises the volume fraction every that many steps
    static vector<EulerReducedStateVector> solve(vector<EulerReducedStateVector>& initialCells, double cellSpacing,
                                                 double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                 int subcyclingIterations, int reinitialisationFrequency,
                                                 EulerMaterialParameters material1Parameters,
                                                 EulerMaterialParameters material2Parameters);
    static vector<vector<EulerReducedStateVector> > solve2D(vector<vector<EulerReducedStateVector> >& initialCells,
                                                            double cellSpacing, double CFLCoefficient, double finalTime,
                                                            double bias, int slopeLimiter, int subcyclingIterations,
                                                            int reinitialisationFrequency,
                                                            EulerMaterialParameters material1Parameters,
                                                            EulerMaterialParameters material2Parameters);
    // the multiphysics two-material model (Solvers/secondordersolver.cpp:314-350, :430-468), exact form
    static vector<EulerMultiphysicsStateVector> solve(vector<EulerMultiphysicsStateVector>& initialCells, double cellSpacing,
                                                      double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                      int subcyclingIterations, int reinitialisationFrequency,
                                                      EulerMaterialParameters material1Parameters,
                                                      EulerMaterialParameters material2Parameters);
    static vector<vector<EulerMultiphysicsStateVector> > solve2D(vector<vector<EulerMultiphysicsStateVector> >& initialCells,
                                                                 double cellSpacing, double CFLCoefficient, double finalTime,
                                                                 double bias, int slopeLimiter, int subcyclingIterations,
                                                                 int reinitialisationFrequency,
                                                                 EulerMaterialParameters material1Parameters,
                                                                 EulerMaterialParameters material2Parameters);
    // step-count overloads (not in the reference): also stop after maxSteps steps when maxSteps > 0
    static vector<EulerReducedStateVector> solve(vector<EulerReducedStateVector>& initialCells, double cellSpacing,
                                                 double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                 int subcyclingIterations, int reinitialisationFrequency,
                                                 EulerMaterialParameters material1Parameters,
                                                 EulerMaterialParameters material2Parameters, int maxSteps);
    static vector<vector<EulerReducedStateVector> > solve2D(vector<vector<EulerReducedStateVector> >& initialCells,
                                                            double cellSpacing, double CFLCoefficient, double finalTime,
                                                            double bias, int slopeLimiter, int subcyclingIterations,
                                                            int reinitialisationFrequency,
                                                            EulerMaterialParameters material1Parameters,
                                                            EulerMaterialParameters material2Parameters, int maxSteps);
    static vector<EulerStateVector> solve(vector<EulerStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                          double finalTime, double bias, int slopeLimiter, int subcyclingIterations,
                                          EulerMaterialParameters mp, int maxSteps);
    static vector<vector<EulerStateVector> > solve2D(vector<vector<EulerStateVector> >& initialCells, double cellSpacing,
                                                     double CFLCofficient, double finalTime, double bias, int slopeLimiter,
                                                     int subcyclingIterations, EulerMaterialParameters mp, int maxSteps);
};

class MHDSecondOrderSolver {
public:
    static void computeXSLICTimeStep2D(vector<vector<MHDStateVector> >& currentCells,
                                       vector<vector<MHDStateVector> >& currentCellsWithBoundary, double cellSpacing,
                                       double timeStep, double bias, int slopeLimiter, MHDMaterialParameters mp);
    static void computeYSLICTimeStep2D(vector<vector<MHDStateVector> >& currentCells,
                                       vector<vector<MHDStateVector> >& currentCellsWithBoundary, double cellSpacing,
                                       double timeStep, double bias, int slopeLimiter, MHDMaterialParameters mp);
    static vector<MHDStateVector> solve(vector<MHDStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, double bias, int slopeLimiter, int subcyclingIterations,
                                        MHDMaterialParameters mp);
    static vector<vector<MHDStateVector> > solve2D(vector<vector<MHDStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                   int subcyclingIterations, MHDMaterialParameters mp);
    static vector<MHDStateVector> solve(vector<MHDStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, double bias, int slopeLimiter, int subcyclingIterations,
                                        MHDMaterialParameters mp, int maxSteps);
    static vector<vector<MHDStateVector> > solve2D(vector<vector<MHDStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                   int subcyclingIterations, MHDMaterialParameters mp, int maxSteps);
    // the MHD reduced two-material model (Solvers/mhdsecondordersolver.cpp:445-495, :615-675): c_h of both materials
    // set every step, RK4 GLM damping sub-cycles, reinitialisation every reinitialisationFrequency steps; exact form
    static vector<MHDReducedStateVector> solve(vector<MHDReducedStateVector>& initialCells, double cellSpacing,
                                               double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                               int subcyclingIterations, int reinitialisationFrequency,
                                               MHDMaterialParameters material1Parameters,
                                               MHDMaterialParameters material2Parameters);
    static vector<vector<MHDReducedStateVector> > solve2D(vector<vector<MHDReducedStateVector> >& initialCells,
                                                          double cellSpacing, double CFLCoefficient, double finalTime,
                                                          double bias, int slopeLimiter, int subcyclingIterations,
                                                          int reinitialisationFrequency,
                                                          MHDMaterialParameters material1Parameters,
                                                          MHDMaterialParameters material2Parameters);
    static vector<MHDReducedStateVector> solve(vector<MHDReducedStateVector>& initialCells, double cellSpacing,
                                               double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                               int subcyclingIterations, int reinitialisationFrequency,
                                               MHDMaterialParameters material1Parameters,
                                               MHDMaterialParameters material2Parameters, int maxSteps);
    static vector<vector<MHDReducedStateVector> > solve2D(vector<vector<MHDReducedStateVector> >& initialCells,
                                                          double cellSpacing, double CFLCoefficient, double finalTime,
                                                          double bias, int slopeLimiter, int subcyclingIterations,
                                                          int reinitialisationFrequency,
                                                          MHDMaterialParameters material1Parameters,
                                                          MHDMaterialParameters material2Parameters, int maxSteps);
    // the MHD multiphysics two-material model, 1D (Solvers/mhdsecondordersolver.cpp:362-385): no source, no
    // reinitialisation, each material's c_h as given; exact form; maxSteps > 0 also stops after that many steps
    static vector<MHDMultiphysicsStateVector> solve(vector<MHDMultiphysicsStateVector>& initialCells,
                                                    double cellSpacing, double CFLCoefficient, double finalTime,
                                                    double bias, int slopeLimiter, int subcyclingIterations,
                                                    int reinitialisationFrequency,
                                                    MHDMaterialParameters material1Parameters,
                                                    MHDMaterialParameters material2Parameters, int maxSteps = 0);
    // the MHD intermediate two-material model (Solvers/mhdsecondordersolver.cpp:387-440, :552-...), exact form; 2D
    // with mirror ghosts on every side (the reference's own 2D padding of this model misfills its outermost bottom row)
    static vector<MHDIntermediateStateVector> solve(vector<MHDIntermediateStateVector>& initialCells,
                                                    double cellSpacing, double CFLCoefficient, double finalTime,
                                                    double bias, int slopeLimiter, int subcyclingIterations,
                                                    int reinitialisationFrequency,
                                                    MHDMaterialParameters material1Parameters,
                                                    MHDMaterialParameters material2Parameters);
    static vector<vector<MHDIntermediateStateVector> > solve2D(vector<vector<MHDIntermediateStateVector> >& initialCells,
                                                               double cellSpacing, double CFLCoefficient,
                                                               double finalTime, double bias, int slopeLimiter,
                                                               int subcyclingIterations, int reinitialisationFrequency,
                                                               MHDMaterialParameters material1Parameters,
                                                               MHDMaterialParameters material2Parameters);
};

// FirstOrderSolver / MHDFirstOrderSolver / HPRFirstOrderSolver::solve{,2D} (Solvers/firstordersolver.h:86-97,
// Solvers/mhdfirstordersolver.h:77-90, Solvers/hprfirstordersolver.h:77-90): FORCE of the cells themselves over a
// 1-ghost boundary; subcyclingIterations is accepted and, as in the reference, does nothing.  The maxSteps
// overloads (not in the reference) also stop after that many steps.
class FirstOrderSolver {
public:
    static vector<EulerStateVector> solve(vector<EulerStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                          double finalTime, int subcyclingIterations, EulerMaterialParameters mp);
    static vector<vector<EulerStateVector> > solve2D(vector<vector<EulerStateVector> >& initialCells, double cellSpacing,
                                                     double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                     EulerMaterialParameters mp);
    static vector<EulerStateVector> solve(vector<EulerStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                          double finalTime, int subcyclingIterations, EulerMaterialParameters mp, int maxSteps);
    static vector<vector<EulerStateVector> > solve2D(vector<vector<EulerStateVector> >& initialCells, double cellSpacing,
                                                     double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                     EulerMaterialParameters mp, int maxSteps);
};

class MHDFirstOrderSolver {
public:
    // the MHD multiphysics model, 1D (Solvers/mhdfirstordersolver.cpp:480-…); maxSteps > 0 also stops after that
    // many steps (not in the reference)
    static vector<MHDMultiphysicsStateVector> solve(vector<MHDMultiphysicsStateVector>& initialCells, double cellSpacing,
                                                    double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                    MHDMaterialParameters material1Parameters,
                                                    MHDMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<MHDStateVector> solve(vector<MHDStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, int subcyclingIterations, MHDMaterialParameters mp);
    static vector<vector<MHDStateVector> > solve2D(vector<vector<MHDStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                   MHDMaterialParameters mp);
    static vector<MHDStateVector> solve(vector<MHDStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, int subcyclingIterations, MHDMaterialParameters mp, int maxSteps);
    static vector<vector<MHDStateVector> > solve2D(vector<vector<MHDStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                   MHDMaterialParameters mp, int maxSteps);
};

class HPRFirstOrderSolver {
public:
    // the HPR two-material models (Solvers/hprfirstordersolver.cpp:501-546, :576-638), exact form; maxSteps > 0 also
    // stops after that many steps (not in the reference)
    static vector<HPRReducedStateVector> solve(vector<HPRReducedStateVector>& initialCells, double cellSpacing,
                                               double CFLCoefficient, double finalTime, int subcyclingIterations,
                                               HPRMaterialParameters material1Parameters,
                                               HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<vector<HPRReducedStateVector> > solve2D(vector<vector<HPRReducedStateVector> >& initialCells,
                                                          double cellSpacing, double CFLCoefficient, double finalTime,
                                                          int subcyclingIterations,
                                                          HPRMaterialParameters material1Parameters,
                                                          HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<HPRIntermediateStateVector> solve(vector<HPRIntermediateStateVector>& initialCells, double cellSpacing,
                                                    double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                    HPRMaterialParameters material1Parameters,
                                                    HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<vector<HPRIntermediateStateVector> > solve2D(vector<vector<HPRIntermediateStateVector> >& initialCells,
                                                               double cellSpacing, double CFLCoefficient,
                                                               double finalTime, int subcyclingIterations,
                                                               HPRMaterialParameters material1Parameters,
                                                               HPRMaterialParameters material2Parameters,
                                                               int maxSteps = 0);
    static vector<HPRMultiphysicsStateVector> solve(vector<HPRMultiphysicsStateVector>& initialCells, double cellSpacing,
                                                    double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                    HPRMaterialParameters material1Parameters,
                                                    HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<HPRStateVector> solve(vector<HPRStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, int subcyclingIterations, HPRMaterialParameters mp);
    static vector<vector<HPRStateVector> > solve2D(vector<vector<HPRStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                   HPRMaterialParameters mp);
    static vector<HPRStateVector> solve(vector<HPRStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, int subcyclingIterations, HPRMaterialParameters mp, int maxSteps);
    static vector<vector<HPRStateVector> > solve2D(vector<vector<HPRStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, int subcyclingIterations,
                                                   HPRMaterialParameters mp, int maxSteps);
};

class HPRSecondOrderSolver {
public:
    static vector<HPRStateVector> solve(vector<HPRStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, double bias, int slopeLimiter, int subcyclingIterations,
                                        HPRMaterialParameters mp);
    static vector<vector<HPRStateVector> > solve2D(vector<vector<HPRStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                   int subcyclingIterations, HPRMaterialParameters mp);
    static vector<HPRStateVector> solve(vector<HPRStateVector>& initialCells, double cellSpacing, double CFLCoefficient,
                                        double finalTime, double bias, int slopeLimiter, int subcyclingIterations,
                                        HPRMaterialParameters mp, int maxSteps);
    static vector<vector<HPRStateVector> > solve2D(vector<vector<HPRStateVector> >& initialCells, double cellSpacing,
                                                   double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                                   int subcyclingIterations, HPRMaterialParameters mp, int maxSteps);
    // the HPR two-material models (Solvers/hprsecondordersolver.cpp:402-500, :548-658): RK4 relaxation sub-cycles
    // around the sweeps, reinitialisation every reinitialisationFrequency steps; exact form; maxSteps > 0 also stops
    // after that many steps (not in the reference)
    static vector<HPRReducedStateVector> solve(vector<HPRReducedStateVector>& initialCells, double cellSpacing,
                                               double CFLCoefficient, double finalTime, double bias, int slopeLimiter,
                                               int subcyclingIterations, int reinitialisationFrequency,
                                               HPRMaterialParameters material1Parameters,
                                               HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<vector<HPRReducedStateVector> > solve2D(vector<vector<HPRReducedStateVector> >& initialCells,
                                                          double cellSpacing, double CFLCoefficient, double finalTime,
                                                          double bias, int slopeLimiter, int subcyclingIterations,
                                                          int reinitialisationFrequency,
                                                          HPRMaterialParameters material1Parameters,
                                                          HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<HPRIntermediateStateVector> solve(vector<HPRIntermediateStateVector>& initialCells, double cellSpacing,
                                                    double CFLCoefficient, double finalTime, double bias,
                                                    int slopeLimiter, int subcyclingIterations,
                                                    int reinitialisationFrequency,
                                                    HPRMaterialParameters material1Parameters,
                                                    HPRMaterialParameters material2Parameters, int maxSteps = 0);
    static vector<vector<HPRIntermediateStateVector> > solve2D(vector<vector<HPRIntermediateStateVector> >& initialCells,
                                                               double cellSpacing, double CFLCoefficient,
                                                               double finalTime, double bias, int slopeLimiter,
                                                               int subcyclingIterations, int reinitialisationFrequency,
                                                               HPRMaterialParameters material1Parameters,
                                                               HPRMaterialParameters material2Parameters,
                                                               int maxSteps = 0);
    // the HPR multiphysics model, 1D (Solvers/hprsecondordersolver.cpp:354-400; its sub-cycle loops are empty)
    static vector<HPRMultiphysicsStateVector> solve(vector<HPRMultiphysicsStateVector>& initialCells, double cellSpacing,
                                                    double CFLCoefficient, double finalTime, double bias,
                                                    int slopeLimiter, int subcyclingIterations,
                                                    int reinitialisationFrequency,
                                                    HPRMaterialParameters material1Parameters,
                                                    HPRMaterialParameters material2Parameters, int maxSteps = 0);
};
