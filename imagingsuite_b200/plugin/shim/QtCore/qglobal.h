/* The two export macros the MuhRec headers take from Qt (<QtCore/qglobal.h>); a MuhRec build
 * with Qt uses Qt's own header instead. On Linux both expand to nothing. */
#pragma once
#define Q_DECL_EXPORT
#define Q_DECL_IMPORT
