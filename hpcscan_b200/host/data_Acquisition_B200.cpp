#include "data_Acquisition_B200.h"

#include <cmath>
#include <string>

#include "config.h"
#include "grid_B200.h"
#include "output_report.h"

namespace hpcscan {

namespace {
bool ok(int rc, const char* caller)
{
	if (rc == B200_OK) return true;
	printError((std::string("IN ") + caller + ", " + b200_last_error()).c_str());
	return false;
}
} // namespace

DataAcquisition_B200::~DataAcquisition_B200(void)
{
	if (d_rec) b200_free(d_rec);
	if (d_trace) b200_free(d_trace);
}

Rtn_code DataAcquisition_B200::initialize(DataAcqui_type acquiType, Grid& coefGrid, Myint ntIn)
{
	if (DataAcquisition::initialize(acquiType, coefGrid, ntIn) != RTN_CODE_OK) return RTN_CODE_KO;
	const size_t nr = size_t(nRecLoc > 0 ? nRecLoc : 0);
	if (nr == 0) return RTN_CODE_OK;
	if (!ok(b200_malloc(&d_rec, nr * sizeof(Myint64)), "DataAcquisition_B200::initialize")) return RTN_CODE_KO;
	if (!ok(b200_memcpy_h2d(d_rec, tab_recIdxLoc, nr * sizeof(Myint64), nullptr), "DataAcquisition_B200::initialize"))
		return RTN_CODE_KO;
	const size_t bytes = nr * size_t(nt) * sizeof(Myfloat);
	if (!ok(b200_malloc(&d_trace, bytes), "DataAcquisition_B200::initialize")) return RTN_CODE_KO;
	if (!ok(b200_memset(d_trace, 0, bytes, nullptr), "DataAcquisition_B200::initialize")) return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "DataAcquisition_B200::initialize") ? RTN_CODE_OK : RTN_CODE_KO;
}

Rtn_code DataAcquisition_B200::recordTrace(Grid& grid, Modeling_type modType, Myint it, Myfloat dt)
{
	if (modType != FORWARD) return DataAcquisition::recordTrace(grid, modType, it, dt);
	Grid_B200* g = dynamic_cast<Grid_B200*>(&grid);
	if (!g) {
		printError("IN DataAcquisition_B200::recordTrace, the grid is not a B200 grid");
		return RTN_CODE_KO;
	}
	const double t0 = MPI_Wtime();
	if (nSrc != 0) {
		// the Ricker sample appliSourceTerm assigned on the host: f0 = freqMax / 2.5,
		// t0 = 1.5 sqrt(6) / (pi f0), in FP64, stored as Myfloat
		const Myfloat64 f0 = Config::Instance()->freqMax / 2.5;
		const Myfloat64 t00 = 1.5 * sqrt(6.) / (M_PI * f0);
		const Myfloat64 tt = it * dt;
		const Myfloat64 tau = M_PI * f0 * (tt - t00);
		const Myfloat64 a2 = pow(tau, 2.);
		const Myfloat sample = (1. - 2. * a2) * exp(-a2);
		if (!ok(b200_set_point(g->field(), srcIdx[0], sample, nullptr), "DataAcquisition_B200::recordTrace"))
			return RTN_CODE_KO;
		g->markDeviceWritten();
	}
	if (nRecLoc > 0) {
		void* out = static_cast<char*>(d_trace) + size_t(it) * sizeof(Myfloat);
		if (!ok(b200_gather_points(g->field(), static_cast<const int64_t*>(d_rec), nRecLoc, out, nt, nullptr),
					"DataAcquisition_B200::recordTrace"))
			return RTN_CODE_KO;
	}
	if (!ok(b200_stream_sync(nullptr), "DataAcquisition_B200::recordTrace")) return RTN_CODE_KO;
	record_trace_time = MPI_Wtime() - t0;
	return RTN_CODE_OK;
}

Rtn_code DataAcquisition_B200::writeTrace(std::string fileName)
{
	if (nRecLoc > 0 &&
			!ok(b200_memcpy_d2h(trace, d_trace, size_t(nRecLoc) * size_t(nt) * sizeof(Myfloat), nullptr),
				"DataAcquisition_B200::writeTrace"))
		return RTN_CODE_KO;
	if (!ok(b200_stream_sync(nullptr), "DataAcquisition_B200::writeTrace")) return RTN_CODE_KO;
	return DataAcquisition::writeTrace(fileName);
}

} // namespace hpcscan
