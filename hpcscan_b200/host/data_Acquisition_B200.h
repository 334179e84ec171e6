//-------------------------------------------------------------------------------------------------------
// DataAcquisition_B200: sources and receivers of hpcscan's Modeling test case on a B200 grid.
//
// hpcscan's DataAcquisition::appliSourceTerm is not virtual and writes the source sample into the
// grid's host array (src/data_Acquisition.cpp:286-320), which the device wavefield never sees.
// recordTrace (virtual, called in the same time step after the snapshots) therefore writes the
// same Ricker sample into the device wavefield first (assignment, as appliSourceTerm does), then
// gathers the receivers on the device into a device trace buffer; writeTrace brings the traces
// back to the base class's host buffer and writes them in hpcscan's format.
//-------------------------------------------------------------------------------------------------------

#ifndef HPCSCAN_DATA_ACQUISITION_B200_H_
#define HPCSCAN_DATA_ACQUISITION_B200_H_

#include <string>

#include "data_Acquisition.h"

namespace hpcscan {

class DataAcquisition_B200 : public DataAcquisition
{
public:
	DataAcquisition_B200(void) {}
	~DataAcquisition_B200(void);

	virtual Rtn_code initialize(DataAcqui_type acquiType, Grid& coefGrid, Myint nt);
	virtual Rtn_code recordTrace(Grid& grid, Modeling_type modType, Myint it, Myfloat dt);
	virtual Rtn_code writeTrace(std::string fileName);

private:
	void* d_rec = nullptr;      // receiver indices (device)
	void* d_trace = nullptr;    // traces, receiver-major as the base class keeps them (device)
};

} // namespace hpcscan

#endif
