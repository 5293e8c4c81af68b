// Stand-in for range-model-lib's REigenValueSolverConf (TEST INFRASTRUCTURE): the method and the
// three numbers REigenValueSolver reads from it (src/reigenvaluesolver.cpp).
#ifndef REF_SHIM_RML_EIGEN_VALUE_SOLVER_CONF_H
#define REF_SHIM_RML_EIGEN_VALUE_SOLVER_CONF_H

#include "rbl_utils.h"

class REigenValueSolverConf
{
    public:
        enum Method { Lanczos = 0, Arnoldi, Rayleigh };

        Method method = Lanczos;

    protected:
        uint nEigenValues = 1;
        uint nIterations = 1;
        double solverCvgValue = 1e-6;

    public:
        uint getNEigenValues() const { return nEigenValues; }
        void setNEigenValues(uint n) { nEigenValues = n; }
        uint getNIterations() const { return nIterations; }
        void setNIterations(uint n) { nIterations = n; }
        double getSolverCvgValue() const { return solverCvgValue; }
        void setSolverCvgValue(double v) { solverCvgValue = v; }
};

#endif
