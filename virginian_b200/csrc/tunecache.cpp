/*
 * Persistent cache of tuned launch shapes.
 *
 * The tuners (virg_gpu_query_tune, autotuned batches) time candidate shapes
 * per program-shape key; the winners are kept in the engine and appended to
 * a text file so later processes start with them:
 *
 *   $VIRGINIAN_B200_TUNE_CACHE        the file; set but empty: no file
 *   else $XDG_CACHE_HOME/virginian_b200/shapes.txt
 *   else $HOME/.cache/virginian_b200/shapes.txt
 *
 * A line is "<build>|<device>|<key>\t<threads> <stage_kb> <stages> <ctas>
 * <chunk_rows> <full_mode>".  <build> is this library's build stamp, so a
 * rebuilt kernel (whose best shapes may differ) ignores older lines;
 * <device> is the device's name and SM count.  Lines are appended with one
 * write each, so processes that tune at the same time interleave whole
 * lines; the last line for a key wins when the file is read.
 */
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "vgpu_engine.h"
#include "engine_internal.h"

namespace vgpu {

namespace {

const char kBuildStamp[] = __DATE__ " " __TIME__;

std::string cache_path()
{
	if (const char *p = getenv("VIRGINIAN_B200_TUNE_CACHE"))
		return p;
	const char *xdg = getenv("XDG_CACHE_HOME");
	if (xdg && *xdg)
		return std::string(xdg) + "/virginian_b200/shapes.txt";
	const char *home = getenv("HOME");
	if (home && *home)
		return std::string(home) + "/.cache/virginian_b200/shapes.txt";
	return "";
}

std::string line_prefix(const virg_gpu_engine *e)
{
	return std::string(kBuildStamp) + "|" + e->device_name + "/" + std::to_string(e->nsm) + "|";
}

/* mkdir -p of the file's directory */
void make_dirs(const std::string &file)
{
	for (size_t i = 1; i < file.size(); i++)
		if (file[i] == '/')
			mkdir(file.substr(0, i).c_str(), 0755);
}

}  // namespace

void tune_cache_load(virg_gpu_engine *e)
{
	const std::string path = cache_path();
	if (path.empty())
		return;
	FILE *f = fopen(path.c_str(), "r");
	if (!f)
		return;
	const std::string pre = line_prefix(e);
	char buf[1024];
	while (fgets(buf, sizeof(buf), f)) {
		if (strncmp(buf, pre.c_str(), pre.size()) != 0)
			continue;
		char *tab = strchr(buf + pre.size(), '\t');
		if (!tab)
			continue;
		Shape s;
		if (sscanf(tab + 1, "%u %u %u %u %u %u", &s.threads, &s.stage_kb, &s.stages, &s.ctas_per_sm, &s.chunk_rows,
				&s.full_mode) != 6 || !shape_supported(s))
			continue;
		e->tuned[std::string(buf + pre.size(), tab)] = s;
	}
	fclose(f);
}

void tune_remember(virg_gpu_engine *e, const std::string &key, const Shape &s)
{
	e->tuned[key] = s;
	const std::string path = cache_path();
	if (path.empty() || key.find('\n') != std::string::npos || key.find('\t') != std::string::npos)
		return;
	make_dirs(path);
	const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_APPEND, 0644);
	if (fd < 0)
		return;  /* the cache is an optimisation: an unwritable file only costs re-tuning */
	char tail[128];
	snprintf(tail, sizeof(tail), "\t%u %u %u %u %u %u\n", s.threads, s.stage_kb, s.stages, s.ctas_per_sm, s.chunk_rows,
		s.full_mode);
	const std::string line = line_prefix(e) + key + tail;
	if (write(fd, line.data(), line.size()) < 0) {
		/* nothing to undo: the shape stays in the engine */
	}
	close(fd);
}

}  // namespace vgpu
