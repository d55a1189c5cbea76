#pragma once
/**
 * @file SimulationConfig.hpp
 * @brief Simulation parameters read from the reference's JSON schema
 *        (include/SimulationConfig.hpp:37-195 of tobjec/parallel-critical-collapse):
 *        the same keys, defaults (DebugNx 100, DebugNtau 1) and null handling.
 */
#include "common.hpp"

struct SimulationConfig {
    size_t Ntau;
    real_t Dim;
    real_t XLeft, XMid, XRight;
    real_t EpsNewton, PrecisionNewton, SlowError;
    int MaxIterNewton;
    bool Verbose, Debug, Converged;
    size_t NLeft, NRight, DebugNx, DebugNtau;
    real_t PrecisionIRK;
    Scheme SchemeIRK;
    int MaxIterIRK;
    real_t Delta = 0.0;
    bool IRKPredictor = false;  // extension key "IRKPredictor" (see pcc_solve_desc::irk_predictor)
    bool ShootBothSides = false;  // extension key "ShootBothSides" (see pcc_solve_desc::shoot_both_sides)
    vec_real fc, psic, Up;

    explicit SimulationConfig(json in)
    {
        Ntau = in["Ntau"];
        Dim = in["Dim"];
        XLeft = in["XLeft"];
        XMid = in["XMid"];
        XRight = in["XRight"];
        EpsNewton = in["EpsNewton"];
        PrecisionNewton = in["PrecisionNewton"];
        SlowError = in["SlowError"];
        MaxIterNewton = in["MaxIterNewton"];
        if (in.contains("IRKPredictor") && !in["IRKPredictor"].is_null()) IRKPredictor = in["IRKPredictor"];
        if (in.contains("ShootBothSides") && !in["ShootBothSides"].is_null()) ShootBothSides = in["ShootBothSides"];
        Verbose = in["Verbose"];
        Debug = in["Debug"];
        Converged = in["Converged"];
        NLeft = in["NLeft"];
        NRight = in["NRight"];
        PrecisionIRK = in["PrecisionIRK"];
        MaxIterIRK = in["MaxIterIRK"];
        switch (in["SchemeIRK"].get<int>()) {
            case 1: SchemeIRK = Scheme::IRK1; break;
            case 2: SchemeIRK = Scheme::IRK2; break;
            case 3: SchemeIRK = Scheme::IRK3; break;
            default: throw std::invalid_argument("Wrong IRK Scheme stage supplied!");
        }
        DebugNx = (in.contains("DebugNx") && !in["DebugNx"].is_null()) ? in["DebugNx"].get<size_t>() : 100;
        DebugNtau = (in.contains("DebugNtau") && !in["DebugNtau"].is_null()) ? in["DebugNtau"].get<size_t>() : 1;
        const json& ic = in["Initial_Conditions"];
        if (!ic["Delta"].is_null()) Delta = ic["Delta"];
        if (!ic["fc"].is_null()) fc = ic["fc"].get<vec_real>();
        if (!ic["psic"].is_null()) psic = ic["psic"].get<vec_real>();
        if (!ic["Up"].is_null()) Up = ic["Up"].get<vec_real>();
    }

    static SimulationConfig loadFromJson(const std::string& filename)
    {
        std::ifstream in(filename);
        if (!in) throw std::runtime_error("Could not open config file: " + filename);
        json j;
        in >> j;
        return SimulationConfig(j);
    }

    static void saveToJson(const std::string& filename, json& simRes)
    {
        std::ofstream file(filename);
        file << simRes;
    }

    /// The numeric part the C ABI consumes.
    pcc_solve_desc desc() const
    {
        pcc_solve_desc d{};
        d.ntau = (int)Ntau;
        d.dim = Dim;
        d.xl = XLeft;
        d.xm = XMid;
        d.xr = XRight;
        d.eps_newton = EpsNewton;
        d.nl = (int)NLeft;
        d.nr = (int)NRight;
        d.prec_irk = PrecisionIRK;
        d.scheme = int(SchemeIRK) + 1;
        d.max_irk = MaxIterIRK;
        d.prec_newton = PrecisionNewton;
        d.slow_error = SlowError;
        d.max_newton = MaxIterNewton;
        d.irk_predictor = IRKPredictor ? 1 : 0;
        d.shoot_both_sides = ShootBothSides ? 1 : 0;
        return d;
    }

    void print_config() const
    {
        std::cout << "Simulation configuration:\n"
                  << "Ntau: " << Ntau << "\nDim: " << Dim << "\nXLeft: " << XLeft << "\nXMid: " << XMid
                  << "\nXRight: " << XRight << "\nEpsNewton: " << EpsNewton << "\nPrecisionNewton: " << PrecisionNewton
                  << "\nSlowError: " << SlowError << "\nMaxIterNewton: " << MaxIterNewton << "\nVerbose: " << Verbose
                  << "\nDebug: " << Debug << "\nDebugNx: " << DebugNx << "\nDebugNtau: " << DebugNtau
                  << "\nConverged: " << Converged << "\nNLeft: " << NLeft << "\nNRight: " << NRight
                  << "\nSchemeIRK: " << int(SchemeIRK) + 1 << "\nPrecisionIRK: " << PrecisionIRK
                  << "\nMaxIterIRK: " << MaxIterIRK << "\nDelta: " << Delta << "\nfc is not empty: " << !fc.empty()
                  << "\npsic is not empty: " << !psic.empty() << "\nUp is not empty: " << !Up.empty() << std::endl;
    }
};
