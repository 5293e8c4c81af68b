// Stand-in for range-model-lib's RMatrixSolverConf (TEST INFRASTRUCTURE): the fields
// src/rmatrixsolver.cpp reads, set by the driver.
#ifndef REF_SHIM_RML_MATRIX_SOLVER_CONF_H
#define REF_SHIM_RML_MATRIX_SOLVER_CONF_H

#include <QString>

#include "rbl_utils.h"

class RMatrixSolverConf
{
    public:
        enum Type { None = 0, CG, GMRES, NTypes };

    protected:
        Type type = CG;
        uint nOuterIterations = 1000;
        uint nInnerIterations = 30;
        double solverCvgValue = 1.0e-5;
        uint outputFrequency = 1;
        QString outputFileName;

    public:
        RMatrixSolverConf() = default;
        explicit RMatrixSolverConf(Type type) : type(type) {}

        Type getType() const { return type; }
        void setType(Type t) { type = t; }
        uint getNOuterIterations() const { return nOuterIterations; }
        void setNOuterIterations(uint n) { nOuterIterations = n; }
        uint getNInnerIterations() const { return nInnerIterations; }
        void setNInnerIterations(uint n) { nInnerIterations = n; }
        double getSolverCvgValue() const { return solverCvgValue; }
        void setSolverCvgValue(double v) { solverCvgValue = v; }
        uint getOutputFrequency() const { return outputFrequency; }
        void setOutputFrequency(uint f) { outputFrequency = f; }
        const QString &getOutputFileName() const { return outputFileName; }
        void setOutputFileName(const QString &f) { outputFileName = f; }

        static QString getName(Type t)
        {
            switch (t) {
                case CG: return QString("Conjugate Gradient");
                case GMRES: return QString("Generalized Minimal Residual");
                default: return QString("None");
            }
        }
};

#endif
