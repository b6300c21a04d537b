// migration.exe parameters.txt -- drop-in for src/migration_main.cpp.
//
// Reads the same keys (src/migration/migration.cu:9-23): a random boundary of
// int(mig_rbc_length/dh)+1 cells with mig_rbc_ratio / mig_rbc_varVp, the shot
// data {mig_input_folder}{mig_input_prefix}{s+1}.bin, and writes
// {mig_output_folder}RTM_section_{int(fmax)}Hz_{nz}x{nx}x{ny}_{int(dh)}m.bin
// (export_seismic, migration.cu:90-117).
// Optional keys: b200_batch (shots per launch), b200_seed (random-boundary
// seed of shot s is b200_seed + s; the reference seeds from the clock),
// b200_fixes (default 1: remove the source while rebuilding the forward
// field; 0: keep it, as the reference does).
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
        const float ratio = fwh::param_f(pf, "mig_rbc_ratio");
        const float varVp = fwh::param_f(pf, "mig_rbc_varVp");
        const float length = fwh::param_f(pf, "mig_rbc_length");
        const std::string in_folder = fwh::param(pf, "mig_input_folder");
        const std::string in_prefix = fwh::param(pf, "mig_input_prefix");
        const std::string out_folder = fwh::param(pf, "mig_output_folder");
        const int batch = std::max(1, fwh::opt_i(pf, "b200_batch", 1));
        const int seed = fwh::opt_i(pf, "b200_seed", 1);
        const int flags = fwh::opt_i(pf, "b200_fixes", 1) ? FWI_FLAG_SUBTRACT_SOURCE : 0;
        const int nb = fwh::pad_cells(length, m.dh);
        fwi_ctx *ctx = fwh::make_context(m, nb, FWI_BOUNDARY_RBC, 0.0f, batch, flags);
        fwh::check(fwi_set_velocity(ctx, m.vp.data()), ctx, "fwi_set_velocity");
        std::cout << fwh::banner("Reverse Time Migration");

        fwh::Clock clock;
        const size_t per_shot = (size_t)m.nt * m.rec.n;
        // every shot gets its own random boundary (seed b200_seed + s), built
        // per batch slot, so `batch` shots with different pads share a launch
        const fwi_rbc rbc{0, ratio, varVp, 0.98f};
        fwh::check(fwi_set_shot_random_boundary(ctx, &rbc, (uint64_t)seed), ctx, "random boundary");
        std::vector<float> data(per_shot * batch);
        std::vector<int> ids(batch);
        for (int s0 = 0; s0 < m.src.n; s0 += batch) {
            const int n = std::min(batch, m.src.n - s0);
            for (int k = 0; k < n; ++k) {
                const int s = s0 + k;
                std::cout << "Running shot " << s + 1 << " of " << m.src.n << " in total\n";
                ids[k] = s;
                fwh::read_binary(in_folder + in_prefix + std::to_string(s + 1) + ".bin", data.data() + k * per_shot,
                                 per_shot);
            }
            fwh::check(fwi_rtm_shots(ctx, ids.data(), n, data.data()), ctx, "fwi_rtm_shots");
        }
        const double secs = clock.seconds();
        std::vector<float> image((size_t)m.nz * m.nx * m.ny);
        fwh::check(fwi_rtm_image(ctx, image.data()), ctx, "fwi_rtm_image");
        const std::string file = out_folder + "RTM_section_" + std::to_string(int(m.fmax)) + "Hz_" +
                                 std::to_string(m.nz) + "x" + std::to_string(m.nx) + "x" + std::to_string(m.ny) +
                                 "_" + std::to_string((int)m.dh) + "m.bin";
        fwh::write_binary(file, image.data(), image.size());
        std::cout << "\nRun time: " << secs << " s." << std::endl;
        fwi_destroy(ctx);
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    return 0;
}
