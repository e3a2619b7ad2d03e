// The reference's particle snapshot files (GOTPM build).
//
// jwrite (Cosmos/CosmosRW/kjhrw.c:169-216) writes, per rank, an ASCII header
// of "define <key> = <value>" lines from FILE_HEADER (Params/params.h:500-517,
// printed by write_head, Params/header.c:28-31) closed by
// "#End of Ascii Header", then the raw particle records: DM_NP dark-matter
// records (dmparticletype, 32 bytes, or treedmparticletype, 40 bytes, by the
// header's "Particle Type"), then the SPH, star and AGN records, then the
// SimParameters struct itself. jread (kjhrw.c:51-150) reads the header with
// read_head (Params/header.c:72-104), matching each line against the same key
// formats with sscanf, then the records; when the trailing struct is missing
// it redoes the domain decomposition instead.
//
// Here the header is parsed by key, the dark-matter records are read as they
// lie in the file, and files are written with the reference's key formats
// (so read_head recognises every line) and the dark-matter records only: no
// SPH, star or AGN particles and no trailing struct, which is the form jread
// handles by decomposing the domain itself. FILE_HEADER has no Rsphere line:
// the cut is a run parameter (params.dat), not part of a snapshot.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <stdlib.h>

#include <string>

#include "tpm_engine.h"

namespace tpm {
void set_last_error(const char *msg);
}

namespace {

const char *kClosing = "#End of Ascii Header";

int err(int code, const std::string &msg) {
  tpm::set_last_error(msg.c_str());
  return code;
}

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\0')) a++;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\n' || s[b - 1] == '\r' || s[b - 1] == '\0')) b--;
  return s.substr(a, b - a);
}

// One header line "define <key> = <value> [# comment]": key and the value's
// first token.
bool parse_line(const std::string &line, std::string &key, std::string &val) {
  if (line.compare(0, 7, "define ") != 0) return false;
  size_t eq = line.find(" = ", 7);
  if (eq == std::string::npos) return false;
  key = trim(line.substr(7, eq - 7));
  std::string rest = line.substr(eq + 3);
  size_t e = 0;
  while (e < rest.size() && rest[e] != ' ' && rest[e] != '\t' && rest[e] != '\n' && rest[e] != '#') e++;
  val = rest.substr(0, e);
  return true;
}

// The reference's key formats for the lines this writer emits
// (Params/params.h:38-139); the padding is part of each key.
const char *kStarting = "#Start of the Ascii Header of the GOTPM Simulation\n";
const char *kNull = "##################################################\n";

}  // namespace

extern "C" {

int tpm_snapshot_info_read(const char *path, tpm_snapshot_info *info) {
  if (!path || !info) return err(TPM_E_ARG, "NULL argument");
  FILE *fp = fopen(path, "rb");
  if (!fp) return err(TPM_E_ARG, std::string("cannot open ") + path);
  memset(info, 0, sizeof(*info));
  info->ptype = -1;
  std::string line;
  bool closed = false;
  int c;
  while (!closed) {
    line.clear();
    while ((c = fgetc(fp)) != EOF) {
      line.push_back((char)c);
      if (c == '\n') break;
    }
    if (line.empty()) break;
    if (line.compare(0, strlen(kClosing), kClosing) == 0) {
      closed = true;
      break;
    }
    std::string k, v;
    if (!parse_line(line, k, v)) continue;
    double d = atof(v.c_str());
    long long l = atoll(v.c_str());
    if (k == "Nx") info->nx = l;
    else if (k == "Ny") info->ny = l;
    else if (k == "Nz") info->nz = l;
    else if (k == "DNp") info->np_dm = l;
    else if (k == "BNp") info->np_sph = l;
    else if (k == "SNp") info->np_star = l;
    else if (k == "ANp") info->np_agn = l;
    else if (k == "Particle Type") info->ptype = (int32_t)l;
    else if (k == "OmegaMatter0") info->omep = (float)d;
    else if (k == "OmegaLambda0") info->omeplam = (float)d;
    else if (k == "w0(eos of DE)") info->wlam0 = (float)d;
    else if (k == "wa(eos of DE)") info->wlam1 = (float)d;
    else if (k == "Amax") info->amax = (float)d;
    else if (k == "Anow") info->anow = d;
    else if (k == "Astep") info->astep = d;
    else if (k == "Theta") info->theta = (float)d;
    else if (k == "EPSILON") info->epsilon = (float)d;
    else if (k == "Rsphere") info->rsphere = (float)d;
    else if (k == "Boxsize(Mpc/h)") info->boxsize = (float)d;
    else if (k == "Stepcount") info->stepcount = (int32_t)l;
  }
  long off = ftell(fp);
  fclose(fp);
  if (!closed) return err(TPM_E_ARG, std::string(path) + ": no '#End of Ascii Header' line");
  if (info->ptype != 0 && info->ptype != 1) return err(TPM_E_ARG, std::string(path) + ": unknown particle type");
  info->record_bytes = info->ptype == 0 ? 32 : 40;
  info->data_offset = off;
  return 0;
}

int tpm_snapshot_read_dm(const char *path, const tpm_snapshot_info *info, void *records, int64_t first,
                         int64_t count) {
  if (!path || !info || (!records && count > 0) || first < 0 || count < 0 || first + count > info->np_dm)
    return err(TPM_E_ARG, "bad arguments to tpm_snapshot_read_dm");
  FILE *fp = fopen(path, "rb");
  if (!fp) return err(TPM_E_ARG, std::string("cannot open ") + path);
  int64_t off = info->data_offset + first * (int64_t)info->record_bytes;
  if (fseek(fp, (long)off, SEEK_SET) != 0) {
    fclose(fp);
    return err(TPM_E_ARG, "seek failed");
  }
  size_t got = fread(records, (size_t)info->record_bytes, (size_t)count, fp);
  fclose(fp);
  if ((int64_t)got != count) return err(TPM_E_ARG, std::string(path) + ": file shorter than its header says");
  return 0;
}

int tpm_snapshot_write(const char *path, const tpm_snapshot_info *info, const void *dm_records) {
  if (!path || !info || (!dm_records && info->np_dm > 0) || (info->ptype != 0 && info->ptype != 1))
    return err(TPM_E_ARG, "bad arguments to tpm_snapshot_write");
  FILE *fp = fopen(path, "wb");
  if (!fp) return err(TPM_E_ARG, std::string("cannot create ") + path);
  // the lines of FILE_HEADER the engine has values for, in its order and with
  // its key formats
  fputs(kStarting, fp);
  fputs(kNull, fp);
  fprintf(fp, "define Myid                = %d # Processor id\n", 0);
  fprintf(fp, "define Nid                 = %d # Number of Processors\n", 1);
  fputs(kNull, fp);
  fprintf(fp, "define OmegaMatter0        = %f # Current Omega Matter\n", info->omep);
  fprintf(fp, "define OmegaLambda0        = %f # Current Omega Lambda\n", info->omeplam);
  fprintf(fp, "define w0(eos of DE)       = %f # w0 of Lambda\n", info->wlam0);
  fprintf(fp, "define wa(eos of DE)       = %f # w1 of Lambda\n", info->wlam1);
  fprintf(fp, "define Boxsize(Mpc/h)      = %f # Simulation Box size in Mpc/h\n", info->boxsize);
  fputs(kNull, fp);
  fprintf(fp, "define Amax                = %f # Maximum expansion factor/ final time\n", info->amax);
  fprintf(fp, "define Anow                = %.17g # Current expansion factor/ current time\n", info->anow);
  fprintf(fp, "define Astep               = %.17g\n", info->astep);
  fprintf(fp, "define Theta               = %f # Current cell opening angle in Tree correction\n", info->theta);
  fprintf(fp, "define EPSILON             = %f # Force Smoothing Length\n", info->epsilon);
  fprintf(fp, "define Nx                  = %lld # Number of grids along x axis\n", (long long)info->nx);
  fprintf(fp, "define Ny                  = %lld # Number of grids along y axis\n", (long long)info->ny);
  fprintf(fp, "define Nz                  = %lld # Number of grids along z axis\n", (long long)info->nz);
  fprintf(fp, "define Stepcount           = %d # Current time step number\n", info->stepcount);
  fprintf(fp, "define Np                  = %lld\n", (long long)info->np_dm);
  fprintf(fp, "define DNp                 = %lld\n", (long long)info->np_dm);
  fprintf(fp, "define BNp                 = %lld\n", 0ll);
  fprintf(fp, "define SNp                 = %lld\n", 0ll);
  fprintf(fp, "define ANp                 = %lld\n", 0ll);
  fprintf(fp, "define Particle Type       = %d\n", info->ptype);
  // FILE_HEADER records sizeof(dmparticletype) here whatever the type
  fprintf(fp, "define Particle_TYPE_Size  = %lu\n", 32ul);
  fputs(kNull, fp);
  fprintf(fp, "%s\n", kClosing);
  size_t rb = info->ptype == 0 ? 32 : 40;
  size_t put = info->np_dm > 0 ? fwrite(dm_records, rb, (size_t)info->np_dm, fp) : 0;
  int bad = ferror(fp);
  fclose(fp);
  if (bad || (int64_t)put != info->np_dm) return err(TPM_E_ARG, std::string("write failed: ") + path);
  return 0;
}

}  // extern "C"
