// inversion.exe parameters.txt -- drop-in for src/inversion_main.cpp.
//
// The reference's FWI loop (src/inversion_main.cpp:13-22, src/inversion/inversion.cu:115-383):
//   compute_gradient   per shot: observed data, modelled data in the Cerjan
//                      grid, residual obs-cal and its squared norm, then (while
//                      iteration <= max_iteration) the gradient through a fresh
//                      random boundary; crop, / illumination, -d2/dz2 below
//                      depth_mask, / max|g|
//   check_convergence  residuo += sqrt(sum res^2)
//   optimization       parabola through steps 0, 0.02 dm, 0.05 dm of the
//                      slowness-squared model, dm = 1/vmin^2 - 1/vmax^2
//   update_model       m -= step g, v = 1/sqrt(m), model_FWI_iteration_{it}_... file
// then convergence_{max_iteration}_iterations.txt and final_model_FWI_... .
//
// By default (b200_fixes = 1) the loop corrects the reference's quirks: it
// uploads the updated model, zeroes the illumination per gradient, keeps
// d2/dy2, removes the source in the rebuild and bounds the line-search step to
// [0, 8 x the largest trial step] (the bound of the Python driver, fwi.py).
// b200_fixes = 0 reproduces the reference
// for parity, quirks included: the device model keeps the 0.05 dm trial model
// after the line search, the illumination accumulates over every gradient,
// there is no d2/dy2 term and no source removal, and the step is unbounded
// except for the CFL check.
// The misfit sums are FP64 on the GPU (the reference sums in FP32 on the host).
#include <fstream>

#include "workflow.hpp"

namespace {

// Largest line-search step as a multiple of the 0.05 dm trial step (the same
// bound as fwi.STEP_BOUND).
constexpr float kStepBound = 8.0f;

struct Inversion {
    std::string pf;
    fwh::Model m;
    fwi_ctx *abc = nullptr, *rbc = nullptr;
    fwi_rbc rbc_recipe{};
    int max_iteration = 0, iteration = 0, seed = 1;
    bool fixes = false;
    float zmask = 0, vmin = 0, vmax = 0;
    std::string in_folder, in_prefix, out_folder, res_folder;
    std::vector<float> model, gradient, v_abc, obs, cal, res;
    std::vector<float> residuo;
    size_t npts = 0, per_shot = 0;

    std::string suffix() const
    {
        return std::to_string(int(m.fmax)) + "Hz_" + std::to_string(m.nz) + "x" + std::to_string(m.nx) + "x" +
               std::to_string(m.ny) + "_" + std::to_string((int)m.dh) + "m.bin";
    }

    // obs - cal for every shot with the ABC context's current velocity; returns
    // sum res^2 and, when `grad` is set, back-propagates each residual.
    double sweep(bool grad)
    {
        double sum = 0.0;
        for (int s = 0; s < m.src.n; ++s) {
            fwh::read_binary(in_folder + in_prefix + std::to_string(s + 1) + ".bin", obs.data(), per_shot);
            fwh::check(fwi_model_shots(abc, &s, 1, cal.data()), abc, "fwi_model_shots");
            double sq = 0.0;
            fwh::check(fwi_residual(abc, obs.data(), cal.data(), (int64_t)per_shot, res.data(), &sq), abc,
                       "fwi_residual");
            sum += sq;
            if (grad) {
                // update_RBC (inversion.cu:204-216): the ABC model, re-padded, new random pad
                fwh::check(fwi_set_velocity(rbc, v_abc.data()), rbc, "fwi_set_velocity");
                fwh::check(fwi_apply_random_boundary(rbc, &rbc_recipe, (uint64_t)(seed + s + 7919 * iteration)),
                           rbc, "random boundary");
                fwh::check(fwi_gradient_shots(rbc, &s, 1, res.data()), rbc, "fwi_gradient_shots");
            }
        }
        return sum;
    }

    void compute_gradient()
    {
        if (fixes)
            fwh::check(fwi_reset_accumulators(rbc), rbc, "reset");
        else
            fwh::check(fwi_zero_image(rbc), rbc, "zero gradient");
        if (iteration == max_iteration) ++iteration;
        const double sum = sweep(iteration <= max_iteration);
        residuo.push_back(sqrtf((float)sum));
        float gmax = 0;
        fwh::check(fwi_gradient_post(rbc, zmask, gradient.data(), &gmax), rbc, "fwi_gradient_post");
    }

    void set_abc_model(const std::vector<float> &v)
    {
        v_abc = v;
        fwh::check(fwi_set_velocity(abc, v_abc.data()), abc, "fwi_set_velocity");
    }

    // linesearch (inversion.cu:315-347): misfit of the trial model m - alpha g.
    float linesearch(float alpha)
    {
        std::vector<float> v(npts);
#pragma omp parallel for
        for (long i = 0; i < (long)npts; ++i) v[i] = 1.0f / sqrtf(model[i] - alpha * gradient[i]);
        set_abc_model(v);
        return sqrtf((float)sweep(false));
    }

    void optimization_and_update()
    {
        const float dm = (1.0f / (vmin * vmin)) - (1.0f / (vmax * vmax));
        const float a0 = 0.00f * dm, a1 = 0.02f * dm, a2 = 0.05f * dm;
        const float f0 = residuo.back();
        const float f1 = linesearch(a1);
        const float f2 = linesearch(a2);
        const float num = (a1 * a1 - a2 * a2) * f0 + (a2 * a2 - a0 * a0) * f1 + (a0 * a0 - a1 * a1) * f2;
        const float den = (a1 - a2) * f0 + (a2 - a0) * f1 + (a0 - a1) * f2;
        float step = 0.5f * (num / den);
        if (fixes) {
            // The reference extrapolates the parabola without bound; with a
            // misfit that falls almost linearly over [0, a2] its vertex lands far
            // outside the bracket and the model leaves the physical range.  Keep
            // the step in [0, 8 a2], and take the best trial step when the
            // parabola is not convex.
            const float slope01 = (f1 - f0) / (a1 - a0), slope12 = (f2 - f1) / (a2 - a1);
            const bool convex = slope12 > slope01;  // positive second divided difference
            if (!convex || !(step > 0)) step = f2 < f1 ? (f2 < f0 ? a2 : 0.0f) : (f1 < f0 ? a1 : 0.0f);
            step = std::min(step, kStepBound * a2);
        }
        std::vector<float> v(npts);
#pragma omp parallel for
        for (long i = 0; i < (long)npts; ++i) {
            model[i] = model[i] - step * gradient[i];
            v[i] = 1.0f / sqrtf(model[i]);
        }
        std::cout << "Iteration " << iteration << ": step " << step << " (misfits " << f0 << ", " << f1 << ", " << f2
                  << ")\n";
        fwh::write_binary(out_folder + "model_FWI_iteration_" + std::to_string(iteration) + "_" + suffix(), v.data(),
                          npts);
        final_v = v;
        if (fixes) set_abc_model(v);  // the reference leaves the 0.05 dm trial model on the device
    }
    std::vector<float> final_v;
};

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " parameters.txt\n";
        return 2;
    }
    Inversion I;
    I.pf = argv[1];
    const std::string &pf = I.pf;
    try {
        I.m = fwh::read_model(pf);
        const float abc_length = fwh::param_f(pf, "abc_length");
        const float abc_factor = fwh::param_f(pf, "abc_factor");
        I.rbc_recipe = fwi_rbc{0, fwh::param_f(pf, "inv_rbc_ratio"), fwh::param_f(pf, "inv_rbc_varVp"), 0.98f};
        const float rbc_length = fwh::param_f(pf, "inv_rbc_length");
        I.zmask = fwh::param_f(pf, "depth_mask");
        I.in_folder = fwh::param(pf, "inv_input_folder");
        I.in_prefix = fwh::param(pf, "inv_input_prefix");
        I.out_folder = fwh::param(pf, "inv_output_folder");
        I.res_folder = fwh::param(pf, "inv_residuo_folder");
        I.max_iteration = fwh::param_i(pf, "max_iteration");
        I.seed = fwh::opt_i(pf, "b200_seed", 1);
        I.fixes = fwh::opt_i(pf, "b200_fixes", 1) != 0;
        const fwh::Model &m = I.m;
        I.npts = (size_t)m.nz * m.nx * m.ny;
        I.per_shot = (size_t)m.nt * m.rec.n;
        I.abc = fwh::make_context(m, fwh::pad_cells(abc_length, m.dh), FWI_BOUNDARY_ABC, abc_factor, 1, 0);
        I.rbc = fwh::make_context(m, fwh::pad_cells(rbc_length, m.dh), FWI_BOUNDARY_RBC, 0.0f, 1,
                                  I.fixes ? (FWI_FLAG_GRAD_DY | FWI_FLAG_SUBTRACT_SOURCE) : 0);
        I.vmin = 1e9f;
        I.vmax = 0.0f;
        for (float v : m.vp) {
            I.vmin = std::min(I.vmin, v);
            I.vmax = std::max(I.vmax, v);
        }
        I.model.resize(I.npts);
        for (size_t i = 0; i < I.npts; ++i) I.model[i] = 1.0f / (m.vp[i] * m.vp[i]);
        I.gradient.assign(I.npts, 0.0f);
        I.obs.resize(I.per_shot);
        I.cal.resize(I.per_shot);
        I.res.resize(I.per_shot);
        I.final_v = m.vp;
        I.set_abc_model(m.vp);
        std::cout << fwh::banner("Full Waveform Inversion");

        fwh::Clock clock;
        for (;;) {
            I.compute_gradient();
            ++I.iteration;  // check_convergence (inversion.cu:280-289)
            std::cout << "Residuo " << I.residuo.size() - 1 << ": " << I.residuo.back() << "\n";
            if (I.iteration > I.max_iteration) break;
            I.optimization_and_update();
        }
        const std::string conv = I.res_folder + "convergence_" + std::to_string(I.max_iteration) + "_iterations.txt";
        std::ofstream f(conv);
        if (!f.is_open()) throw std::invalid_argument("Error: \033[31m" + conv + "\033[0;0m could not be opened!");
        for (int r = 0; r <= I.max_iteration && r < (int)I.residuo.size(); ++r) f << I.residuo[r] << "\n";
        f.close();
        std::cout << "Text file \033[34m" << conv << "\033[0;0m was successfully written." << std::endl;
        fwh::write_binary(I.out_folder + "final_model_FWI_" + I.suffix(), I.final_v.data(), I.npts);
        std::cout << "\nRun time: " << clock.seconds() << " s." << std::endl;
        fwi_destroy(I.abc);
        fwi_destroy(I.rbc);
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    return 0;
}
