// dualgpmf: the command line of the reference's single-precision sampler
// (src/dualgpm.cpp built with DUALRES_SINGLE_PRECISION), running on the GPU
// through the library's C ABI.
//
// Options, defaults and messages follow GPMCommandParser
// (include/dualres/impl/CommandParser/GPMCommandParser.inl:219-606); the
// pipeline follows src/dualgpm.cpp:45-357: read and mask the images, estimate
// the covariance parameters when --covariance is absent, fit, then write
//   <output>_posterior_mean.nii.gz, _posterior_variance.nii.gz,
//   _posterior_activation.nii.gz, _residual.nii.gz
// and with --samples also <output>_samples.dat and <output>_stats.csv.
// Extension: --chains K runs K independent chains and pools them.
#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dualres_b200.h"
#include "nifti.h"

using drb::nifti::Image;

namespace {

struct Options {
  std::string highres, stdres, hmask, smask, omask, output;
  std::vector<float> covariance;
  float neighborhood = -1.f;
  int burnin = 1000, nsave = 1000, thin = 3, leapfrog = 25, threads = 0, chains = 1, device = 0;
  double mhtarget = 0.65;
  unsigned seed = 1;
  bool monitor = false, samples = false, rq = false, help = false;
};

void usage(const std::string& caller) {
  std::cerr << "\nFit dual (or single) resolution Gaussian process model to NIfTI data:\n"
            << "\nUsage:\n\t" << caller << " --highres path/to/img1 <options>\n\n";
}

void help(const std::string& caller) {
  usage(caller);
  std::cerr << "REQUIRED:\n"
            << "\t--highres  path/to/img1   Primary data source\n\n"
            << "Optional:\n"
            << "\t--stdres   path/to/img2   Optional secondary data file\n"
            << "\t--burnin       int        Number of MCMC burnin iterations (1000)\n"
            << "\t--chains       int        Independent chains, pooled (1; GPU build only)\n"
            << "\t--covariance   f1 f2 f3   Covariance parameters (variance, bandwidth, exponent)\n"
            << "\t--debug                   Run a short debug-length MCMC chain\n"
            << "\t--device       int        CUDA device (0; GPU build only)\n"
            << "\t--leapfrog     int        Number of MCMC integrator steps (25)\n"
            << "\t--mhtarget     float      Target metropolis hastings rate (0.65)\n"
            << "\t--monitor                 Monitor MCMC iterations\n"
            << "\t--hmask    path/to/mask   Mask image for --highres input\n"
            << "\t--neighborhood float      N'hood size (mm) for kriging approx\n"
            << "\t--nsave        int        MCMC samples to save in output (1000)\n"
            << "\t--omask    path/to/mask   Mask image to define output space\n"
            << "\t--output   file/basename  Path prefix for output files\n"
            << "\t--rational-quadratic      Rational quadratic covariance function\n"
            << "\t--samples                 Request full MCMC output\n"
            << "\t--smask    path/to/mask   Mask image for --stdres input\n"
            << "\t--seed         int        RNG seed\n"
            << "\t--theta        f1 f2 f3   Alias for --covariance\n"
            << "\t--thin         int        Thinning factor for MCMC samples (3)\n"
            << "\t--threads      int        Number of host threads (set-up work)\n\n"
            << "Outputs: *_posterior_mean.nii.gz, *_posterior_variance.nii.gz,\n"
            << "*_posterior_activation.nii.gz and *_residual.nii.gz; with --samples\n"
            << "also *_samples.dat (one line per saved iteration: mu at the output\n"
            << "voxels, sigma per dataset, tau, log likelihood) and *_stats.csv.\n"
            << std::endl;
}

// Returns 0 ok, 1 error, 2 help.
int parse(int argc, char** argv, Options* o) {
  const std::string caller = [&] {
    std::string s = argv[0];
    const size_t k = s.find_last_of('/');
    return k == std::string::npos ? s : s.substr(k + 1);
  }();
  const auto now = std::chrono::high_resolution_clock::now().time_since_epoch();
  o->seed = std::max((unsigned)std::chrono::duration_cast<std::chrono::milliseconds>(now).count(), 1u);
  o->output = "dualgpm_mcmc_" + std::to_string(o->seed) + "_";
  bool error = argc < 2;
  auto need = [&](int& i, int k, const char* msg) {
    if (i + k < argc) return true;
    std::cerr << msg;
    error = true;
    return false;
  };
  auto posint = [&](int& i, int* dst, const char* msg) {
    if (!need(i, 1, msg)) return;
    try {
      *dst = std::max(std::abs(std::stoi(argv[++i])), 1);
    } catch (...) {
      std::cerr << msg;
      error = true;
    }
  };
  auto nifti_arg = [&](int& i, std::string* dst, const char* name) {
    if (!need(i, 1, (std::string("\nWarning: ") + name + " option requires one argument\n").c_str())) return;
    *dst = argv[++i];
    if (!drb::nifti::is_nifti_file(*dst)) {
      std::cerr << "\nWarning: input file does not appear to conform to the nifti-1 standard\n\t" << *dst << std::endl;
      error = true;
    }
  };
  for (int i = 1; i < argc && !error; i++) {
    const std::string a = argv[i];
    if (a == "-h" || a == "--help") {
      o->help = true;
      break;
    } else if (a == "--burnin") {
      posint(i, &o->burnin, "\nWarning: --burnin option requires 1 positive integer argument\n");
    } else if (a == "--covariance" || a == "--theta") {
      const char* msg = "\nWarning: --covariance option requires 3 numeric arguments\n";
      if (!need(i, 3, msg)) break;
      o->covariance.resize(3);
      for (int j = 0; j < 3; j++) {
        try {
          o->covariance[j] = (float)std::stod(argv[++i]);
        } catch (...) {
          std::cerr << msg;
          error = true;
          break;
        }
      }
    } else if (a == "--debug") {
      o->burnin = 50;
      o->nsave = 10;
      o->thin = 1;
      o->monitor = true;
      o->samples = true;
    } else if (a == "--highres") {
      nifti_arg(i, &o->highres, "--highres");
    } else if (a == "--hmask" || a == "-hm") {
      nifti_arg(i, &o->hmask, "--hmask");
    } else if (a == "--leapfrog" || a == "-L") {
      posint(i, &o->leapfrog, "\nWarning: --leapfrog option requires 1 positive integer argument\n");
    } else if (a == "--mhtarget") {
      const char* msg = "\nWarning: --mhtarget option requires 1 numeric argument on (0, 1)\n";
      if (!need(i, 1, msg)) break;
      try {
        o->mhtarget = std::stod(argv[++i]);
        if (o->mhtarget <= 0 || o->mhtarget >= 1) throw std::domain_error("--mhtarget outside bounds");
      } catch (...) {
        std::cerr << msg;
        error = true;
      }
    } else if (a == "--monitor") {
      o->monitor = true;
    } else if (a == "--neighborhood") {
      const char* msg = "\nWarning: --neighborhood option requires 1 numeric argument\n";
      if (!need(i, 1, msg)) break;
      try {
        o->neighborhood = std::fabs((float)std::stod(argv[++i]));
      } catch (...) {
        std::cerr << msg;
        error = true;
      }
    } else if (a == "--nsave" || a == "-n") {
      posint(i, &o->nsave, "\nWarning: --nsave option requires 1 positive integer argument\n");
    } else if (a == "--output" || a == "-o") {
      if (!need(i, 1, "\nWarning: --output option requires 1 string argument\n")) break;
      o->output = argv[++i];
    } else if (a == "--omask" || a == "-om") {
      nifti_arg(i, &o->omask, "--omask");
    } else if (a == "--rational-quadratic") {
      o->rq = true;
    } else if (a == "--samples") {
      o->samples = true;
    } else if (a == "--seed") {
      const char* msg = "\nWarning: --seed option requires 1 integer argument\n";
      if (!need(i, 1, msg)) break;
      try {
        o->seed = (unsigned)std::abs(std::stoi(argv[++i]));
      } catch (...) {
        std::cerr << msg;
        error = true;
      }
    } else if (a == "--smask" || a == "-sm") {
      nifti_arg(i, &o->smask, "--smask");
    } else if (a == "--stdres") {
      nifti_arg(i, &o->stdres, "--stdres");
    } else if (a == "--thin") {
      posint(i, &o->thin, "\nWarning: --thin option requires 1 positive integer argument\n");
    } else if (a == "--threads") {
      const char* msg = "\nWarning: --threads option requires 1 integer argument\n";
      if (!need(i, 1, msg)) break;
      try {
        o->threads = std::abs(std::stoi(argv[++i]));
      } catch (...) {
        std::cerr << msg;
        error = true;
      }
    } else if (a == "--chains") {
      posint(i, &o->chains, "\nWarning: --chains option requires 1 positive integer argument\n");
    } else if (a == "--device") {
      const char* msg = "\nWarning: --device option requires 1 integer argument\n";
      if (!need(i, 1, msg)) break;
      try {
        o->device = std::abs(std::stoi(argv[++i]));
      } catch (...) {
        std::cerr << msg;
        error = true;
      }
    } else {
      std::cerr << "\nWarning: Unrecognized option: " << a << std::endl;
      error = true;
    }
  }
  if (o->help) {
    help(caller);
    return 2;
  }
  if (o->highres.empty() && !error) {
    std::cerr << "\nError: User must supply the --highres argument\n";
    error = true;
  }
  if (o->hmask.empty()) o->hmask = o->highres;
  if (o->omask.empty()) o->omask = o->highres;
  if (error) {
    usage(caller);
    std::cerr << "\nSee " << caller << " --help for more information\n";
    return 1;
  }
  return 0;
}

bool nonzero(float v) { return !(std::isnan(v) || v == 0.f); }

// apply_mask (nifti_manipulation.inl:75-127): zero where the mask is zero or the image is NaN.
void apply_mask(std::vector<float>& img, const std::vector<float>& mask) {
  for (size_t i = 0; i < img.size(); i++)
    if (mask[i] == 0.f || std::isnan(img[i])) img[i] = 0.f;
}

// emplace_nonzero_data (nifti_manipulation.inl:170-201): consecutive values into
// the image's non-zero, non-NaN voxels, in storage order.
void emplace_nonzero(std::vector<float>& img, const std::vector<float>& vals) {
  size_t j = 0;
  for (size_t i = 0; i < img.size() && j < vals.size(); i++)
    if (nonzero(img[i])) img[i] = vals[j++];
}

void check(int rc) {
  if (rc == DR_OK) return;
  const std::string msg = dr_last_error();
  if (rc == DR_ERR_DOMAIN) throw std::domain_error(msg);
  if (rc == DR_ERR_INVALID) throw std::logic_error(msg);
  throw std::runtime_error(msg);
}

float max_voxel_dim(const Image& im) {
  float m = 0.f;
  for (int j = 0; j < 3; j++) {
    float s = 0.f;
    for (int i = 0; i < 4; i++) s += im.qto_xyz[4 * i + j] * im.qto_xyz[4 * i + j];
    m = std::max(m, std::sqrt(s));
  }
  return m;
}

// compute_covar_parameters_if_needed (src/dualgpm.cpp:375-404).
bool covariance_if_needed(std::vector<float>& theta, const Image& im, int device) {
  if (!theta.empty()) return true;
  std::cout << "Estimating covariance parameters... " << std::flush;
  double th[3] = {1.0, 0.6, 1.5};
  const int rc = dr_estimate_covariance(im.data.data(), im.nx(), im.ny(), im.nz(), im.qto_xyz, device, th);
  if (rc != DR_OK) {
    std::cerr << "Could not estimate covar parameters.\n"
              << "Try re-running with the --covariance argument supplied" << std::endl;
    return false;
  }
  for (int i = 0; i < 3; i++) theta.push_back((float)th[i]);
  std::cout << "Done!" << std::endl;
  return true;
}

bool valid_covariance(const std::vector<float>& th) {
  bool ok = true;
  if (th[0] <= 0) { std::cerr << "First covariance parameter (marginal variance) must be > 0\n"; ok = false; }
  if (th[1] <= 0) { std::cerr << "Second covariance parameter (bandwidth) must be > 0\n"; ok = false; }
  if (th[2] <= 0 || th[2] > 2) { std::cerr << "Third covariance parameter (exponent) must be in (0, 2]\n"; ok = false; }
  return ok;
}

void write_image(const Image& geom, const std::vector<float>& vals, const std::string& path) {
  std::remove(path.c_str());
  drb::nifti::write(geom, vals, path);
  std::cout << path << " written\n";
}

int run(const Options& o) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int threads = o.threads > 0 ? o.threads : std::max(1, (int)(0.8 * hw));
  omp_set_num_threads(threads);
  std::cout << "[dualres running on " << threads << " cores, CUDA device " << o.device << "]" << std::endl;

  const std::string f_act = o.output + "_posterior_activation.nii.gz";
  const std::string f_mean = o.output + "_posterior_mean.nii.gz";
  const std::string f_res = o.output + "_residual.nii.gz";
  const std::string f_samples = o.output + "_samples.dat";
  const std::string f_var = o.output + "_posterior_variance.nii.gz";

  std::ofstream samples_out;
  if (o.samples) samples_out.open(f_samples.c_str());

  Image hr = drb::nifti::read(o.highres);
  std::cout << "High-resolution file: " << o.highres << std::endl;
  Image hmask = drb::nifti::read(o.hmask);
  Image omask = drb::nifti::read(o.omask);
  if (drb::nifti::same_orientation(hr, hmask) && hr.nvox() == hmask.nvox()) {
    apply_mask(hr.data, hmask.data);
    std::cout << "\t[Masked by: " << o.hmask << "]" << std::endl;
  } else {
    std::cerr << "  *** WARNING ***  High-resolution image/mask mismatch. Image not masked" << std::endl;
    throw std::domain_error("Improper mask");
  }
  if (!drb::nifti::same_orientation(hr, omask) || hr.nvox() != omask.nvox()) {
    std::cerr << "  *** WARNING ***  High-resolution/output mask mismatch." << std::endl;
    throw std::domain_error("Improper mask");
  }
  if (o.samples && !samples_out) throw std::runtime_error("Error: will not be able to write output to\n  " + f_samples);

  std::vector<float> theta = o.covariance;
  float neighborhood = o.neighborhood;
  Image sr;
  const bool dual = !o.stdres.empty();
  if (dual) {
    sr = drb::nifti::read(o.stdres);
    std::cout << "Standard-resolution file: " << o.stdres << std::endl;
    if (sr.datatype != hr.datatype)
      throw std::domain_error("Error: " + o.highres + " and " + o.stdres + " have different data types\n");
    if (!o.smask.empty()) {
      Image sm = drb::nifti::read(o.smask);
      if (drb::nifti::same_orientation(sr, sm) && sr.nvox() == sm.nvox()) {
        apply_mask(sr.data, sm.data);
        std::cout << "\t[Masked by: " << o.smask << "]" << std::endl;
      } else {
        std::cerr << "  *** WARNING ***  Standard-resolution image/mask mismatch. Image not masked" << std::endl;
      }
    }
    if (!covariance_if_needed(theta, sr, o.device))
      throw std::runtime_error("Error: could not compute covariance parameters from " + o.stdres + "\n");
    if (neighborhood <= 0) neighborhood = 3 * max_voxel_dim(hr);
    std::cout << "Neighborhood: " << neighborhood << " (mm)\n";
  }
  if (!covariance_if_needed(theta, hr, o.device))
    throw std::runtime_error("Error: could not compute covariance parameters from " + o.highres + "\n");
  if (!valid_covariance(theta)) {
    std::ostringstream ss;
    ss << "Error: covariance parameters are not valid (" << theta[0] << ", " << theta[1] << ", " << theta[2] << ")\n";
    throw std::domain_error(ss.str());
  }
  std::cout << "Covariance parameters: (" << theta[0] << ", " << theta[1] << ", " << theta[2] << ")" << std::endl;
  std::cout << "\nMCMC settings:\n-----------------\nBurnin   = " << o.burnin << "\nNSave    = " << o.nsave
            << "\nThin     = " << o.thin << "\nLeapfrog = " << o.leapfrog << "\n-----------------" << std::endl;

  dr_volume_desc d = {};
  d.nx = hr.nx(); d.ny = hr.ny(); d.nz = hr.nz();
  d.highres = hr.data.data();
  d.qform_hr = hr.qto_xyz;
  d.hmask = hmask.data.data();
  d.omask = omask.data.data();
  if (dual) {
    d.sx = sr.nx(); d.sy = sr.ny(); d.sz = sr.nz();
    d.stdres = sr.data.data();
    d.qform_sr = sr.qto_xyz;
  }
  for (int i = 0; i < 3; i++) d.covariance[i] = theta[i];
  d.covfun = o.rq ? DR_COV_RQ : DR_COV_RBF;
  d.neighborhood = neighborhood;
  d.device = o.device;
  dr_volume* vol = nullptr;
  check(dr_volume_create(&d, &vol));
  dr_volume_info info;
  check(dr_volume_info_get(vol, &info));

  std::cout << "\nFitting model with rmHMC";
  if (dual) std::cout << " and projected neighborhood process approximation";
  std::cout << std::endl;
  dr_hmc_opts ho = {o.burnin, o.nsave, o.thin, o.leapfrog, (float)o.mhtarget, (float)(1.0 / o.leapfrog),
                    (uint64_t)o.seed, o.samples ? 1 : 0};
  dr_chainset* cs = nullptr;
  check(dr_chainset_create(vol, o.chains, &ho, &cs));
  // burn-in, then the timed post-burn-in part (mcmc_summary::sampling_time covers the saving phase).  With
  // --monitor every iteration prints each chain's energy transition, step size and MH ratio, as
  // MultiResParameters::update does (MultiResParameters.h:706-713), one iteration at a time.
  std::vector<dr_chain_stats> mon(o.chains);
  std::vector<int> last_it(o.chains, 0);
  auto monitor_line = [&]() {
    check(dr_chain_stats_get(cs, mon.data()));
    const std::streamsize prec = std::cout.precision();
    for (int c = 0; c < o.chains; c++) {
      const dr_chain_stats& m = mon[c];
      if (m.iteration == last_it[c]) continue;  // a chain that has saved nsave samples no longer moves
      last_it[c] = m.iteration;
      if (o.chains > 1) std::cout << "chain " << c << ": ";
      std::cout << std::setprecision(4) << "Energy Transition (" << m.initial_energy << " -> " << m.proposed_energy
                << ");  step size (" << m.last_eps << ");  MH = (" << std::exp(m.last_log_ratio) << ")"
                << std::endl;
    }
    std::cout.precision(prec);
  };
  if (o.monitor) {
    for (int it = 0; it < o.burnin; it++) {
      check(dr_step(cs, 1));
      monitor_line();
    }
  } else if (o.burnin > 0) {
    check(dr_step(cs, o.burnin));
  }
  const auto t0 = std::chrono::high_resolution_clock::now();
  if (o.monitor) {
    for (;;) {
      check(dr_chain_stats_get(cs, mon.data()));
      bool all_done = true;
      for (const auto& m : mon) all_done = all_done && m.done;
      if (all_done) break;
      check(dr_step(cs, 1));
      monitor_line();
    }
  } else {
    check(dr_run(cs));
  }
  const double sampling_s = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();

  std::vector<dr_chain_stats> st(o.chains);
  check(dr_chain_stats_get(cs, st.data()));
  double mh = 0, eps = 0;
  for (const auto& s : st) { mh += s.mh_rate; eps += s.eps; }
  mh /= o.chains;
  eps /= o.chains;

  const int no = info.n_output;
  std::vector<float> mean(no), var(no), act(no);
  check(dr_summary_get(cs, -1, mean.data(), var.data(), act.data()));

  if (o.samples) {
    // gaussian_process_model.h:149-163: mu at the output voxels, sigma per dataset, tau, log likelihood
    const float tau = std::sqrt(1.0f / (1.0f / theta[0]));
    for (int c = 0; c < o.chains; c++) {
      int n_saved = 0;
      std::vector<float> smp((size_t)o.nsave * no);
      std::vector<double> rec((size_t)o.nsave * 3);
      check(dr_samples_get(cs, c, smp.data(), o.nsave, &n_saved));
      check(dr_sample_records_get(cs, c, rec.data(), o.nsave, &n_saved));
      for (int i = 0; i < n_saved; i++) {
        for (int k = 0; k < no; k++) samples_out << smp[(size_t)i * no + k] << "\t";
        samples_out << (float)rec[3 * i] << "\t";
        if (dual) samples_out << (float)rec[3 * i + 1] << "\t";
        samples_out << tau << "\t" << (float)rec[3 * i + 2];
        if (i < n_saved - 1 || c < o.chains - 1) samples_out << std::endl;
      }
    }
    samples_out.close();
    std::cout << f_samples << " written\n";
  }
  dr_chainset_destroy(cs);
  dr_volume_destroy(vol);

  // outputs through the output mask image, in the reference's order
  std::vector<float> img = omask.data;
  if (f_mean != o.highres) {
    emplace_nonzero(img, mean);
    write_image(omask, img, f_mean);
  } else {
    std::cerr << "  *** WARNING *** posterior mean image would overwrite data. File not written\n";
  }
  emplace_nonzero(img, var);
  write_image(omask, img, f_var);
  emplace_nonzero(img, act);
  write_image(omask, img, f_act);
  // residual: hr - mean where both are non-zero (src/dualgpm.cpp:336-346)
  std::vector<float> neg(no);
  for (int i = 0; i < no; i++) neg[i] = -mean[i];
  emplace_nonzero(img, neg);
  std::vector<float> h = hr.data;
  apply_mask(h, img);
  for (size_t i = 0; i < img.size(); i++) img[i] += h[i];
  apply_mask(img, h);
  write_image(omask, img, f_res);

  std::cout << "Post burnin sampling took " << sampling_s << " (sec)\n"
            << "Metropolis-Hastings rate was " << (mh * 100) << "%\n" << std::endl;
  if (o.samples) {
    std::ofstream s((o.output + "_stats.csv").c_str());
    if (s.is_open()) s << "MHrate,SamplingTime,StepSize\n" << (float)mh << "," << sampling_s << "," << (float)eps << "\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  const int p = parse(argc, argv, &o);
  if (p == 2) return 0;
  if (p == 1) return 1;
  try {
    return run(o);
  } catch (const std::exception& e) {
    std::cerr << "\nException caught with message:\n'" << e.what() << "'\n" << std::endl;
  } catch (...) {
    std::cerr << "\nUnknown error\n" << std::endl;
  }
  return 1;
}
