// modeling.exe parameters.txt -- drop-in for src/modeling_main.cpp.
//
// Same keys, same output files as the reference (src/modeling/modeling.cu:
// 17-34, 83-90, 302-307): one seismogram_nt{nt}_nr{nrec}_{int(1e6 dt)}us_shot_{s+1}.bin
// per shot in mod_output_folder, Fortran [nt, nrec] float32, Cerjan sponge of
// int(abc_length/dh)+1 cells.  Optional key b200_batch: shots per launch.
#include "workflow.hpp"

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " parameters.txt\n";
        return 2;
    }
    const std::string pf = argv[1];
    try {
        fwh::Model m = fwh::read_model(pf);
        const float abc_length = fwh::param_f(pf, "abc_length");
        const float abc_factor = fwh::param_f(pf, "abc_factor");
        const std::string folder = fwh::param(pf, "mod_output_folder");
        const int batch = std::max(1, fwh::opt_i(pf, "b200_batch", 1));
        const int nb = fwh::pad_cells(abc_length, m.dh);
        fwi_ctx *ctx = fwh::make_context(m, nb, FWI_BOUNDARY_ABC, abc_factor, batch, 0);
        fwh::check(fwi_set_velocity(ctx, m.vp.data()), ctx, "fwi_set_velocity");
        std::cout << fwh::banner("Seismic Modeling");
        std::cout << "Model dimensions: (z = " << (m.nz - 1) * m.dh << ", x = " << (m.nx - 1) * m.dh
                  << ", y = " << (m.ny - 1) * m.dh << ") m\n\n";

        fwh::Clock clock;
        const size_t per_shot = (size_t)m.nt * m.rec.n;
        std::vector<float> seis(per_shot * batch);
        for (int s0 = 0; s0 < m.src.n; s0 += batch) {
            const int n = std::min(batch, m.src.n - s0);
            std::vector<int> shots(n);
            for (int k = 0; k < n; ++k) shots[k] = s0 + k;
            std::cout << "Running shots " << s0 + 1 << "-" << s0 + n << " of " << m.src.n << " in total\n";
            fwh::check(fwi_model_shots(ctx, shots.data(), n, seis.data()), ctx, "fwi_model_shots");
            for (int k = 0; k < n; ++k) {
                const std::string file = folder + "seismogram_nt" + std::to_string(m.nt) + "_nr" +
                                         std::to_string(m.rec.n) + "_" + std::to_string(int(1e6f * m.dt)) +
                                         "us_shot_" + std::to_string(s0 + k + 1) + ".bin";
                fwh::write_binary(file, seis.data() + k * per_shot, per_shot);
            }
        }
        std::cout << "\nRun time: " << clock.seconds() << " s." << std::endl;
        fwi_destroy(ctx);
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    return 0;
}
